// C ABI of the library (declared in include/loom_gpu.h).  One translation
// unit: every kernel and host component is included here.
#include "../../include/loom_gpu.h"
#include "prove_flow.cuh"
#include "verify.cuh"

using namespace lg;

namespace lg {
void note_launches(uint64_t k) { g_launches.fetch_add(k); }
}  // namespace lg

struct lg_ctx {
  Ctx c;
  size_t last_proof_len = 0;  // bytes of the last proof in c.proof_buf
};

namespace {

__global__ void k_aos_to_soa(const uint32_t* in, uint64_t n, uint32_t lanes, uint32_t* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n * lanes) return;
  uint64_t row = i / lanes, w = i % lanes;
  out[w * n + row] = in[i];
}
__global__ void k_soa_to_aos(const uint32_t* in, uint64_t n, uint32_t lanes, uint32_t* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n * lanes) return;
  uint64_t row = i / lanes, w = i % lanes;
  out[i] = in[w * n + row];
}

__global__ void k_e6_div_soa(const uint32_t* num, const uint32_t* den, uint64_t n, uint32_t* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  E6 a = ld6(num, n, i), b = ld6(den, n, i);
  st6(out, n, i, e6_mul(a, e6_inv(b)));
}

template <class F> int guarded(lg_ctx* ctx, F f) {
  if (!ctx) return LG_ERR_INVALID;
  try {
    AcctScope acct(&ctx->c.mem);
    LG_CK(cudaSetDevice(ctx->c.device));
    if (ctx->c.stream) {
      LG_CK(cudaStreamSynchronize(ctx->c.stream));
      if (ctx->c.side) LG_CK(cudaStreamSynchronize(ctx->c.side));  // its work reads the arena too
      ctx->c.arena_reset();
      ctx->c.dev_arena.rewind();
    }
    f();
    return LG_OK;
  } catch (Error& e) {
    ctx->c.err = e.what();
    return e.code;
  } catch (std::exception& e) {
    ctx->c.err = e.what();
    return LG_ERR_INVALID;
  }
}

// Copies `words` words from host or device memory into a fresh device buffer.
DBufP to_device(Ctx& c, const uint32_t* src, size_t words, int on_device) {
  auto b = std::make_shared<DBuf>(std::max<size_t>(words, 1), c.stream);
  if (words)
    LG_CK(cudaMemcpyAsync(b->p, src, words * 4, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.stream));
  return b;
}
void from_device(Ctx& c, uint32_t* dst, const uint32_t* src, size_t words, int on_device) {
  LG_CK(cudaMemcpyAsync(dst, src, words * 4, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c.stream));
  LG_CK(cudaStreamSynchronize(c.stream));
}

}  // namespace

extern "C" {

int lg_ctx_create(int device, size_t hbm_budget, lg_ctx** out) {
  if (!out) return LG_ERR_INVALID;
  *out = nullptr;
  lg_ctx* ctx = new lg_ctx();
  ctx->c.device = device;
  ctx->c.mem.budget = (int64_t)hbm_budget;
  int rc = guarded(ctx, [&] {
    LG_CK(cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking));
    LG_CK(cudaStreamCreateWithFlags(&ctx->c.side, cudaStreamNonBlocking));
    LG_CK(cudaEventCreateWithFlags(&ctx->c.fork_ev, cudaEventDisableTiming));
    LG_CK(cudaEventCreateWithFlags(&ctx->c.join_ev, cudaEventDisableTiming));
    LG_CK(cudaEventCreateWithFlags(&ctx->c.upload_ev, cudaEventDisableTiming));
    cudaMemPool_t pool;
    LG_CK(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;  // keep freed blocks for the next prove
    LG_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    LG_CK(cudaDeviceGetAttribute(&ctx->c.sm_count, cudaDevAttrMultiProcessorCount, device));
  });
  if (rc != LG_OK) {
    delete ctx;
    return rc;
  }
  *out = ctx;
  return LG_OK;
}

void lg_ctx_destroy(lg_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->c.device);
  if (ctx->c.stream) cudaStreamSynchronize(ctx->c.stream);
  // every cached device buffer frees on the stream: release them while it exists
  ctx->c.tw.clear();
  ctx->c.tw16.clear();
  ctx->c.tw_split.clear();
  ctx->c.gpow.clear();
  ctx->c.ginvpow.clear();
  ctx->c.cshift.clear();
  ctx->c.lagrange_vals.clear();
  ctx->c.lagrange_coef.clear();
  ctx->c.programs.clear();
  if (ctx->c.stream) {
    cudaStreamSynchronize(ctx->c.stream);
    ctx->c.dev_arena.release(ctx->c.stream);
    cudaStreamSynchronize(ctx->c.stream);
    cudaStreamDestroy(ctx->c.stream);
  }
  if (ctx->c.side) {
    cudaStreamSynchronize(ctx->c.side);
    cudaStreamDestroy(ctx->c.side);
  }
  if (ctx->c.fork_ev) cudaEventDestroy(ctx->c.fork_ev);
  if (ctx->c.join_ev) cudaEventDestroy(ctx->c.join_ev);
  if (ctx->c.upload_ev) cudaEventDestroy(ctx->c.upload_ev);
  if (ctx->c.pinned) cudaFreeHost(ctx->c.pinned);
  delete ctx;
}

int lg_ctx_set_batched(lg_ctx* ctx, int batched) {
  return guarded(ctx, [&] { ctx->c.batched = batched != 0; });
}

int lg_ctx_mem_usage(lg_ctx* ctx, uint64_t* held_bytes, uint64_t* peak_bytes, int reset_peak) {
  if (!ctx) return LG_ERR_INVALID;
  const int64_t h = ctx->c.mem.held.load();
  if (held_bytes) *held_bytes = (uint64_t)std::max<int64_t>(h, 0);
  if (peak_bytes) *peak_bytes = (uint64_t)std::max<int64_t>(ctx->c.mem.peak.load(), 0);
  if (reset_peak) ctx->c.mem.peak.store(h);
  return LG_OK;
}

int lg_device_mem_info(int device, uint64_t* available_bytes, uint64_t* total_bytes) {
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return LG_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) return LG_ERR_CUDA;
  size_t f = 0, t = 0;
  cudaMemPool_t pool;
  uint64_t reserved = 0, used = 0;
  int rc = LG_OK;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess ||
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
    rc = LG_ERR_CUDA;
  cudaSetDevice(prev);
  if (rc != LG_OK) return rc;
  if (available_bytes) *available_bytes = (uint64_t)f + (reserved > used ? reserved - used : 0);
  if (total_bytes) *total_bytes = (uint64_t)t;
  return LG_OK;
}

int lg_mem_info(lg_ctx* ctx, uint64_t* free_bytes, uint64_t* total_bytes) {
  return guarded(ctx, [&] {
    size_t f = 0, t = 0;
    LG_CK(cudaMemGetInfo(&f, &t));
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
  });
}

int lg_ctx_set_leaf_mapping(lg_ctx* ctx, int lanes_per_permutation) {
  return guarded(ctx, [&] {
    if (lanes_per_permutation != 0 && lanes_per_permutation != 1 && lanes_per_permutation != 6)
      throw Error(LG_ERR_INVALID, "leaf mapping must be 0 (auto), 1 or 6 lanes per permutation");
    ctx->c.leaf_mapping = lanes_per_permutation;
  });
}

int lg_ctx_set_tuning(lg_ctx* ctx, const char* name, int64_t value) {
  return guarded(ctx, [&] {
    if (!name) throw Error(LG_ERR_INVALID, "null tuning name");
    std::string n = name;
    auto in = [&](int64_t lo, int64_t hi) {
      if (value < lo || value > hi) throw Error(LG_ERR_INVALID, "tuning " + n + " out of range");
    };
    auto pow2 = [&] {
      if (value & (value - 1)) throw Error(LG_ERR_INVALID, "tuning " + n + " must be a power of two");
    };
    Ctx::Tuning& t = ctx->c.tune;
    if (n == "p2_leaf_min_per_sm") { in(0, 1 << 20); t.p2_leaf_min_per_sm = (uint32_t)value; }
    else if (n == "p2_node_min_per_sm") { in(0, 1 << 20); t.p2_node_min_per_sm = (uint32_t)value; }
    else if (n == "p2_inject_min_per_sm") { in(0, 1 << 20); t.p2_inject_min_per_sm = (uint32_t)value; }
    else if (n == "merkle_tail") { in(2, 1024); pow2(); t.merkle_tail = (uint32_t)value; }
    else if (n == "merkle_subtree") {
      if (value != 0) { in(2, 1024); pow2(); }
      t.merkle_subtree = (uint32_t)value;
    } else if (n == "inject_block") { in(32, 1024); pow2(); t.inject_block = (uint32_t)value; }
    else if (n == "leaf_block") { in(32, 1024); pow2(); t.leaf_block = (uint32_t)value; }
    else if (n == "lde_split") { in(0, 1); t.lde_split = (uint32_t)value; }
    else if (n == "lde_fwd_threads") { in(256, 1024); pow2(); t.lde_fwd_threads = (uint32_t)value; }
    else if (n == "fri_tail_leaves") {
      if (value != 0) { in(2, 1 << 16); pow2(); }
      t.fri_tail_leaves = (uint32_t)value;
    }
    else if (n == "quotient_jit") {
      in(0, 1);
      t.quotient_jit = (uint32_t)value;
    }
    else if (n == "upload_split") { in(0, 1); t.upload_split = (uint32_t)value; }
    else throw Error(LG_ERR_INVALID, "unknown tuning " + n);
  });
}

int lg_ctx_get_tuning(lg_ctx* ctx, const char* name, int64_t* value) {
  return guarded(ctx, [&] {
    if (!name || !value) throw Error(LG_ERR_INVALID, "null argument");
    std::string n = name;
    const Ctx::Tuning& t = ctx->c.tune;
    if (n == "p2_leaf_min_per_sm") *value = t.p2_leaf_min_per_sm;
    else if (n == "p2_node_min_per_sm") *value = t.p2_node_min_per_sm;
    else if (n == "p2_inject_min_per_sm") *value = t.p2_inject_min_per_sm;
    else if (n == "merkle_tail") *value = t.merkle_tail;
    else if (n == "merkle_subtree") *value = t.merkle_subtree;
    else if (n == "inject_block") *value = t.inject_block;
    else if (n == "leaf_block") *value = t.leaf_block;
    else if (n == "lde_split") *value = t.lde_split;
    else if (n == "lde_fwd_threads") *value = t.lde_fwd_threads;
    else if (n == "fri_tail_leaves") *value = t.fri_tail_leaves;
    else if (n == "quotient_jit") *value = t.quotient_jit;
    else if (n == "upload_split") *value = t.upload_split;
    else throw Error(LG_ERR_INVALID, "unknown tuning " + n);
  });
}

const char* lg_last_error(lg_ctx* ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }

int lg_prove(lg_ctx* ctx, const char* hash_backend, const uint32_t* program, size_t program_words,
             const uint32_t* const* witness, int witness_on_device, uint32_t num_queries, uint8_t* proof,
             size_t* proof_len) {
  return guarded(ctx, [&] {
    std::string hb = hash_backend ? hash_backend : "";
    if (hb != "" && hb != "poseidon2")
      throw Error(LG_ERR_UNSUPPORTED, "hash backend \"" + hb + "\" is not available on the GPU path (poseidon2 only)");
    if (!program || !proof_len) throw Error(LG_ERR_INVALID, "null argument");
    Prover pr(ctx->c, program, program_words, num_queries);
    ctx->last_proof_len = 0;
    bool direct = false;
    size_t need = pr.prove(witness, witness_on_device != 0, proof, proof ? *proof_len : 0, &direct);
    *proof_len = need;
    if (!direct) {  // did not fit: kept for lg_last_proof
      ctx->last_proof_len = need;
      throw Error(LG_ERR_BUFFER, "proof buffer too small");
    }
  });
}

int lg_setup(lg_ctx* ctx, const uint32_t* program, size_t program_words, const uint32_t* const* setup_cols,
             int on_device, uint32_t root[8]) {
  return guarded(ctx, [&] {
    if (!program || !setup_cols || !root) throw Error(LG_ERR_INVALID, "null argument");
    Prover pr(ctx->c, program, program_words, 1);
    pr.precommit(setup_cols, on_device != 0);
    LG_CK(cudaStreamSynchronize(ctx->c.stream));
    memcpy(root, pr.prog->setup->root.v, 32);
  });
}

int lg_verify(lg_ctx* ctx, const uint32_t* program, size_t program_words, const uint8_t* proof, size_t proof_len,
              uint32_t num_queries, const uint32_t* setup_root, const char* buses) {
  return guarded(ctx, [&] {
    if (!program || !proof) throw Error(LG_ERR_INVALID, "null argument");
    ArenaScope arena(&ctx->c.dev_arena);
    ProofVerifier v(ctx->c, program, program_words, num_queries);
    Digest root{};
    if (setup_root) memcpy(root.v, setup_root, 32);
    v.verify(proof, proof_len, setup_root ? &root : nullptr, buses);
  });
}

int lg_last_proof(lg_ctx* ctx, uint8_t* proof, size_t* proof_len) {
  if (!ctx || !proof_len) return LG_ERR_INVALID;
  size_t need = ctx->last_proof_len;
  if (!proof || *proof_len < need) { *proof_len = need; return LG_ERR_BUFFER; }
  memcpy(proof, ctx->c.proof_buf.data(), need);
  *proof_len = need;
  return LG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- handles
// Every handle starts with a tag, so lg_release takes any of them.
constexpr uint32_t LG_HANDLE_MAGIC = 0x4c474844u;  // "LGHD"
enum : uint32_t { HK_COMMITTED = 1, HK_SESSION = 2 };

struct lg_committed {
  uint32_t magic = LG_HANDLE_MAGIC, kind = HK_COMMITTED;
  lg_ctx* ctx = nullptr;
  Committed cm;                // LDE, coefficients and tree on the device (shared buffers)
  std::vector<uint32_t> nb, ne;  // per group, declaration order
};

struct lg_session {
  uint32_t magic = LG_HANDLE_MAGIC, kind = HK_SESSION;
  lg_ctx* ctx = nullptr;
  std::unique_ptr<Prover> pr;
};

namespace {

// Groups of a batch given as PCS.Commit's columns (internal/fri/pcs.go:145-168):
// rows[g] Lagrange rows, n_base[g] base columns then n_ext[g] extension
// columns (ext.E6 rows, 6 words each) in `cols`, group by group.  Extension
// columns are laid out as six lanes on the device.
std::vector<GroupSpec> batch_groups(Ctx& c, uint32_t n_groups, const uint64_t* rows, const uint32_t* n_base,
                                    const uint32_t* n_ext, const uint32_t* const* cols, int on_device,
                                    std::vector<DBufP>& keep) {
  if (!n_groups || !rows || !n_base || !n_ext || !cols) throw Error(LG_ERR_INVALID, "null argument");
  std::vector<GroupSpec> gs;
  size_t ci = 0;
  for (uint32_t g = 0; g < n_groups; g++) {
    uint64_t n = rows[g];
    if (n < 2 || (n & (n - 1))) throw Error(LG_ERR_INVALID, "group rows must be a power of two >= 2");
    GroupSpec s;
    s.log_n = 0;
    while ((1ull << s.log_n) < n) s.log_n++;
    s.nb = n_base[g];
    s.ne = n_ext[g];
    s.from_coeffs = false;
    for (uint32_t i = 0; i < s.nb; i++) {
      if (!cols[ci]) throw Error(LG_ERR_INVALID, "null column");
      auto b = to_device(c, cols[ci++], n, on_device);
      s.lanes.push_back(b->p);
      keep.push_back(b);
    }
    for (uint32_t i = 0; i < s.ne; i++) {
      if (!cols[ci]) throw Error(LG_ERR_INVALID, "null column");
      auto a = to_device(c, cols[ci++], 6 * n, on_device);
      auto b = std::make_shared<DBuf>(6 * n, c.stream);
      k_aos_to_soa<<<(unsigned)((6 * n + 255) / 256), 256, 0, c.stream>>>(a->p, n, 6, b->p);
      LG_LAUNCH();
      for (int w = 0; w < 6; w++) s.lanes.push_back(b->p + (size_t)w * n);
      keep.push_back(a);
      keep.push_back(b);
    }
    gs.push_back(s);
  }
  return gs;
}

lg_committed* as_committed(const void* h) {
  auto* c = (lg_committed*)h;
  if (!c || c->magic != LG_HANDLE_MAGIC || c->kind != HK_COMMITTED) return nullptr;
  return c;
}
lg_session* as_session(const void* h) {
  auto* s = (lg_session*)h;
  if (!s || s->magic != LG_HANDLE_MAGIC || s->kind != HK_SESSION) return nullptr;
  return s;
}
// Runs one phase of a session: the context's guard (status codes, device,
// idle stream) with the session's prover; phases allocate from the
// context's memory pool only (no per-call arena), so what one phase leaves
// on the device stays valid for the next.
template <class F> int session_phase(lg_session* s, F f) {
  if (!as_session(s) || !s->pr) return LG_ERR_INVALID;
  return guarded(s->ctx, [&] {
    ArenaScope pool_only(nullptr);
    f(*s->pr);
  });
}

}  // namespace

extern "C" {

int lg_commit_root(lg_ctx* ctx, uint32_t n_groups, const uint64_t* rows, const uint32_t* n_base,
                   const uint32_t* n_ext, const uint32_t* const* cols, int on_device, uint32_t root[8]) {
  return guarded(ctx, [&] {
    if (!root) throw Error(LG_ERR_INVALID, "null argument");
    std::vector<DBufP> keep;
    std::vector<GroupSpec> gs = batch_groups(ctx->c, n_groups, rows, n_base, n_ext, cols, on_device, keep);
    Committed cm = commit(ctx->c, gs, false);
    memcpy(root, cm.tree.root.v, 32);
  });
}

int lg_commit(lg_ctx* ctx, uint32_t n_groups, const uint64_t* rows, const uint32_t* n_base, const uint32_t* n_ext,
              const uint32_t* const* cols, int on_device, lg_committed** out, uint32_t root[8]) {
  if (out) *out = nullptr;
  return guarded(ctx, [&] {
    if (!root || !out) throw Error(LG_ERR_INVALID, "null argument");
    ArenaScope pool_only(nullptr);  // everything here outlives the call
    std::vector<DBufP> keep;
    std::vector<GroupSpec> gs = batch_groups(ctx->c, n_groups, rows, n_base, n_ext, cols, on_device, keep);
    auto h = std::make_unique<lg_committed>();
    h->ctx = ctx;
    h->cm = commit(ctx->c, gs, true);
    for (auto& g : gs) { h->nb.push_back(g.nb); h->ne.push_back(g.ne); }
    memcpy(root, h->cm.tree.root.v, 32);
    LG_CK(cudaStreamSynchronize(ctx->c.stream));
    *out = h.release();
  });
}

int lg_committed_eval(lg_ctx* ctx, const lg_committed* batch, const uint32_t zeta[6], uint32_t n_shifts,
                      const int32_t* shifts, uint32_t* out) {
  return guarded(ctx, [&] {
    const lg_committed* h = as_committed(batch);
    if (!h || !zeta || !out || (n_shifts && !shifts)) throw Error(LG_ERR_INVALID, "null or invalid argument");
    if (h->ctx != ctx) throw Error(LG_ERR_INVALID, "handle belongs to another context");
    Ctx& c = ctx->c;
    ArenaScope arena(&c.dev_arena);
    auto zd = upload_vec(c, std::vector<uint32_t>(zeta, zeta + 6));
    std::vector<DotJob> jobs;
    std::vector<DBufP> keep;
    std::map<std::pair<uint32_t, int32_t>, const uint32_t*> zp;
    for (size_t g = 0; g < h->cm.groups.size(); g++) {
      const LdeOut& l = h->cm.groups[g];
      if (!l.coef) throw Error(LG_ERR_UNSUPPORTED, "this batch keeps no coefficients");
      const size_t n = (size_t)1 << l.log_n;
      for (uint32_t si = 0; si < n_shifts; si++) {
        auto key = std::make_pair(l.log_n, shifts[si]);
        if (!zp.count(key)) {
          const int64_t e = ((int64_t)shifts[si] % (int64_t)n + (int64_t)n) % (int64_t)n;
          const uint32_t ws = mont_pow(root_of_unity_mont((int)l.log_n), (uint64_t)e);
          auto b = std::make_shared<DBuf>(6 * n, c.stream);
          k_e6_powers<<<(unsigned)((n + 127) / 128), 128, 0, c.stream>>>(zd->p, ws, (uint32_t)n, b->p);
          LG_LAUNCH();
          keep.push_back(b);
          zp[key] = b->p;
        }
      }
    }
    // one dot product per (group, polynomial lane, shift)
    for (size_t g = 0; g < h->cm.groups.size(); g++) {
      const LdeOut& l = h->cm.groups[g];
      const uint32_t n = 1u << l.log_n;
      for (uint32_t lane = 0; lane < l.lanes; lane++)
        for (uint32_t si = 0; si < n_shifts; si++)
          jobs.push_back(DotJob{l.coef->p + (size_t)lane * n, zp.at({l.log_n, shifts[si]}), n, (uint32_t)jobs.size()});
    }
    std::vector<uint32_t> dots(6 * jobs.size());
    if (!jobs.empty()) {
      auto jd = upload_vec(c, jobs);
      auto od = std::make_shared<DBuf>(6 * jobs.size(), c.stream);
      k_dot<<<(unsigned)jobs.size(), 256, 0, c.stream>>>((const DotJob*)jd->p, od->p);
      LG_LAUNCH();
      uint32_t* hst = c.host_staging(dots.size());
      c.d2h(hst, od->p, dots.size());
      memcpy(dots.data(), hst, dots.size() * 4);
    }
    // per group: base polynomials, then extension polynomials (their six
    // lanes' values recombined on the E6 basis), each at every shift
    size_t j = 0, o = 0;
    for (size_t g = 0; g < h->cm.groups.size(); g++) {
      const uint32_t nb = h->nb[g], ne = h->ne[g];
      for (uint32_t i = 0; i < nb; i++)
        for (uint32_t si = 0; si < n_shifts; si++, j++, o++)
          for (int q = 0; q < 6; q++) out[6 * o + q] = dots[6 * j + q];
      for (uint32_t i = 0; i < ne; i++) {
        std::vector<E6> acc(n_shifts, e6_zero());
        for (uint32_t w = 0; w < 6; w++)
          for (uint32_t si = 0; si < n_shifts; si++, j++) {
            E6 d, basis = e6_zero();
            for (int q = 0; q < 6; q++) d.c[q] = dots[6 * j + q];
            basis.c[w] = MONT_ONE;
            acc[si] = e6_add(acc[si], e6_mul(d, basis));
          }
        for (uint32_t si = 0; si < n_shifts; si++, o++)
          for (int q = 0; q < 6; q++) out[6 * o + q] = acc[si].c[q];
      }
    }
  });
}

int lg_open_batches(lg_ctx* ctx, uint32_t n_batches, const lg_committed* const* batches, const uint32_t* positions,
                    uint32_t n_positions, uint8_t* out, size_t* out_len) {
  return guarded(ctx, [&] {
    if (!batches || !positions || !out_len || !n_batches || !n_positions) throw Error(LG_ERR_INVALID, "null or empty argument");
    Ctx& c = ctx->c;
    ArenaScope arena(&c.dev_arena);
    std::vector<OpenBatch> obs;
    for (uint32_t b = 0; b < n_batches; b++) {
      const lg_committed* h = as_committed(batches[b]);
      if (!h) throw Error(LG_ERR_INVALID, "not a committed-batch handle");
      if (h->ctx != ctx) throw Error(LG_ERR_INVALID, "handle belongs to another context");
      obs.push_back(OpenBatch{&h->cm, h->nb, h->ne});
    }
    std::vector<uint32_t> pos(positions, positions + n_positions);
    for (uint32_t s : pos)
      if (s >= (1u << LOG_N_FRI)) throw Error(LG_ERR_INVALID, "query position out of range");
    OpenPlan OP;
    const SectionSrc sec = OP.batches_section(obs, n_positions);
    const size_t need = 4 * (size_t)n_positions * sec.q_words;
    if (!out || *out_len < need) {
      *out_len = need;
      throw Error(LG_ERR_BUFFER, "output buffer too small");
    }
    const uint32_t* A = OP.run(c, pos);
    memcpy(out, A + sec.out_off, need);
    *out_len = need;
  });
}

// ---------------------------------------------------------------- sessions
int lg_session_begin(lg_ctx* ctx, const char* hash_backend, const uint32_t* program, size_t program_words,
                     const uint32_t* const* witness, int witness_on_device, uint32_t num_queries, lg_session** out) {
  if (out) *out = nullptr;
  return guarded(ctx, [&] {
    std::string hb = hash_backend ? hash_backend : "";
    if (hb != "" && hb != "poseidon2")
      throw Error(LG_ERR_UNSUPPORTED, "hash backend \"" + hb + "\" is not available on the GPU path (poseidon2 only)");
    if (!program || !out) throw Error(LG_ERR_INVALID, "null argument");
    ArenaScope pool_only(nullptr);
    auto s = std::make_unique<lg_session>();
    s->ctx = ctx;
    s->pr = std::make_unique<Prover>(ctx->c, program, program_words, num_queries);
    s->pr->c.phase_start();
    s->pr->begin(witness, witness_on_device != 0);
    LG_CK(cudaStreamSynchronize(ctx->c.stream));
    *out = s.release();
  });
}

int lg_session_setup_root(lg_session* s, uint32_t root[8], int* has_root) {
  return session_phase(s, [&](Prover& p) {
    if (!root || !has_root) throw Error(LG_ERR_INVALID, "null argument");
    *has_root = p.has_setup_tree() ? 1 : 0;
    if (*has_root) memcpy(root, p.prog->setup->root.v, 32);
  });
}

int lg_session_challenge(lg_session* s, const char* name, const uint32_t digest[8]) {
  return session_phase(s, [&](Prover& p) {
    if (!name || !digest) throw Error(LG_ERR_INVALID, "null argument");
    p.set_challenge(name, digest);
  });
}

int lg_commit_round(lg_session* s, uint32_t round, uint32_t root[8], int* committed, uint32_t* exposed,
                    uint32_t* n_exposed) {
  return session_phase(s, [&](Prover& p) {
    if (!root || !committed || !n_exposed) throw Error(LG_ERR_INVALID, "null argument");
    Digest d{};
    *committed = p.commit_round(round, &d) ? 1 : 0;
    memcpy(root, d.v, 32);
    const std::vector<E6> ev = p.round_exposed(round);
    const uint32_t cap = *n_exposed;
    *n_exposed = (uint32_t)ev.size();
    if (ev.size() > cap || (ev.size() && !exposed)) throw Error(LG_ERR_BUFFER, "exposed-value buffer too small");
    for (size_t i = 0; i < ev.size(); i++) memcpy(exposed + 6 * i, ev[i].c, 24);
  });
}

int lg_quotient(lg_session* s, uint32_t root[8], int* committed) {
  return session_phase(s, [&](Prover& p) {
    if (!root || !committed) throw Error(LG_ERR_INVALID, "null argument");
    Digest d{};
    *committed = p.commit_quotient(&d) ? 1 : 0;
    memcpy(root, d.v, 32);
  });
}

int lg_claimed_values(lg_session* s, uint32_t* values, size_t* n_values) {
  return session_phase(s, [&](Prover& p) {
    if (!n_values) throw Error(LG_ERR_INVALID, "null argument");
    if (p.cv.empty()) p.claimed_values();
    const std::vector<E6> v = p.claimed_values_bind_order();
    const size_t cap = *n_values;
    *n_values = v.size();
    if (v.size() > cap || !values) throw Error(LG_ERR_BUFFER, "claimed-value buffer too small");
    for (size_t i = 0; i < v.size(); i++) memcpy(values + 6 * i, v[i].c, 24);
  });
}

int lg_deep(lg_session* s) {
  return session_phase(s, [&](Prover& p) { p.deep_codewords(); });
}

int lg_fri_commit_levels(lg_session* s, uint32_t root[8], uint32_t* n_levels, uint32_t* first_round) {
  return session_phase(s, [&](Prover& p) {
    if (!root || !n_levels || !first_round) throw Error(LG_ERR_INVALID, "null argument");
    const Digest d = p.commit_levels();
    memcpy(root, d.v, 32);
    *n_levels = (uint32_t)p.L;
    *first_round = (uint32_t)p.r0;
  });
}

int lg_fri_fold_round(lg_session* s, uint32_t round, uint32_t root[8], int* committed) {
  return session_phase(s, [&](Prover& p) {
    if (!root || !committed) throw Error(LG_ERR_INVALID, "null argument");
    Digest d{};
    *committed = p.fri_fold_round((int)round, true, &d) ? 1 : 0;
    memcpy(root, d.v, 32);
  });
}

int lg_fri_final(lg_session* s, uint32_t* values, size_t* n_values) {
  return session_phase(s, [&](Prover& p) {
    if (!n_values) throw Error(LG_ERR_INVALID, "null argument");
    if (p.final_poly.empty()) p.read_final_poly();
    const size_t n = p.nj, cap = *n_values;
    *n_values = n;
    if (n > cap || !values) throw Error(LG_ERR_BUFFER, "final-polynomial buffer too small");
    for (size_t i = 0; i < n; i++)
      for (int w = 0; w < 6; w++) values[6 * i + w] = p.final_poly[w * n + i];
  });
}

int lg_open(lg_session* s, const uint32_t* positions, uint32_t n_positions, uint8_t* proof, size_t* proof_len) {
  lg_session* ss = as_session(s);
  if (!ss) return LG_ERR_INVALID;
  return session_phase(s, [&](Prover& p) {
    if (!positions || !proof_len) throw Error(LG_ERR_INVALID, "null argument");
    std::vector<uint32_t> pos(positions, positions + n_positions);
    bool direct = false;
    ss->ctx->last_proof_len = 0;
    size_t need = p.open_and_encode(pos, proof, proof ? *proof_len : 0, &direct);
    *proof_len = need;
    if (!direct) {
      ss->ctx->last_proof_len = need;
      throw Error(LG_ERR_BUFFER, "proof buffer too small");
    }
  });
}

int lg_session_committed(lg_session* s, uint32_t index, lg_committed** out) {
  if (out) *out = nullptr;
  return session_phase(s, [&](Prover& p) {
    if (!out) throw Error(LG_ERR_INVALID, "null argument");
    if (index >= p.committed.size()) throw Error(LG_ERR_INVALID, "no committed batch at this index");
    auto h = std::make_unique<lg_committed>();
    h->ctx = s->ctx;
    h->cm = p.committed[index];
    const auto& T = p.trees[index];
    for (size_t g = 0; g < T.groups.size(); g++) {
      h->nb.push_back((uint32_t)T.groups[g].bcols.size());
      h->ne.push_back((uint32_t)T.groups[g].ecols.size());
      // the AIR batch keeps its coefficients with the quotient chunks
      if (T.air && !h->cm.groups[g].coef) h->cm.groups[g].coef = p.chunk_coef.at(T.groups[g].module);
    }
    *out = h.release();
  });
}

void lg_release(void* handle) {
  if (lg_committed* c = as_committed(handle)) {
    lg_ctx* ctx = c->ctx;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    c->magic = 0;
    delete c;  // device buffers free on the context's stream
    return;
  }
  if (lg_session* s = as_session(handle)) {
    lg_ctx* ctx = s->ctx;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    s->magic = 0;
    delete s;
  }
}

int lg_rs_encode(lg_ctx* ctx, const uint32_t* in, uint64_t n_rows, uint32_t n_cols, uint32_t* out, int on_device) {
  return guarded(ctx, [&] {
    Ctx& c = ctx->c;
    if (!in || !out || n_rows < 2 || (n_rows & (n_rows - 1))) throw Error(LG_ERR_INVALID, "bad arguments");
    uint32_t logn = 0;
    while ((1ull << logn) < n_rows) logn++;
    auto src = to_device(c, in, n_rows * n_cols, on_device);
    std::vector<const uint32_t*> lanes;
    for (uint32_t i = 0; i < n_cols; i++) lanes.push_back(src->p + (size_t)i * n_rows);
    LdeOut l = lde_lanes(c, lanes, logn, false, false);
    from_device(c, out, l.lde->p, (size_t)n_cols * (n_rows << RATE_LOG), on_device);
  });
}

int lg_poseidon2_permute(lg_ctx* ctx, uint32_t* states, uint64_t n_states, int on_device) {
  return guarded(ctx, [&] {
    Ctx& c = ctx->c;
    if (!states) throw Error(LG_ERR_INVALID, "null argument");
    if (!n_states) return;
    auto b = to_device(c, states, 24 * n_states, on_device);
    k_p2_permute<<<(unsigned)((n_states + 19) / 20), 128, 0, c.stream>>>(b->p, n_states);
    LG_LAUNCH();
    from_device(c, states, b->p, 24 * n_states, on_device);
  });
}

int lg_merkle_root(lg_ctx* ctx, const uint32_t* leaves, uint64_t n_leaves, uint32_t n_inj, const uint64_t* inj_widths,
                   const uint32_t* inj, int on_device, uint32_t root[8]) {
  return guarded(ctx, [&] {
    Ctx& c = ctx->c;
    if (!leaves || !root || n_leaves == 0 || (n_leaves & (n_leaves - 1))) throw Error(LG_ERR_INVALID, "bad leaves");
    if (n_inj && (!inj_widths || !inj)) throw Error(LG_ERR_INVALID, "null injections");
    // the schedule merkle.NewWithInjections accepts (validateInjections,
    // internal/merkle/tree.go:140-160):
    // powers of two, none wider than the leaves, widths never increasing
    for (uint32_t k = 0; k < n_inj; k++) {
      const uint64_t w = inj_widths[k];
      if (w == 0 || (w & (w - 1)) || w > n_leaves || (k && w > inj_widths[k - 1]))
        throw Error(LG_ERR_INVALID, "bad injection schedule");
    }
    TreeDev t;
    while ((1ull << t.log_leaves) < n_leaves) t.log_leaves++;
    t.nodes = std::make_shared<DBuf>(16 * n_leaves, c.stream);
    LG_CK(cudaMemcpyAsync(t.nodes->p + 8 * n_leaves, leaves, 32 * n_leaves,
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.stream));
    size_t off = 0;
    for (uint32_t k = 0; k < n_inj; k++) {
      const uint64_t w = inj_widths[k];
      t.inj.push_back(to_device(c, inj + off, 8 * w, on_device));
      uint32_t lw = 0;
      while ((1ull << lw) < w) lw++;
      t.inj_log_w.push_back(lw);
      off += 8 * w;
    }
    build_tree(c, t);
    memcpy(root, t.root.v, 32);
  });
}

int lg_fri_fold(lg_ctx* ctx, const uint32_t* layer, uint64_t n, const uint32_t alpha[6], uint32_t* out, int on_device) {
  return guarded(ctx, [&] {
    Ctx& c = ctx->c;
    if (!layer || !out || !alpha || n < 2 || (n & (n - 1)) || n > (1ull << 24)) throw Error(LG_ERR_INVALID, "bad arguments");
    int logn = 0;
    while ((1ull << logn) < n) logn++;
    auto a = to_device(c, layer, 6 * n, on_device);
    auto soa = std::make_shared<DBuf>(6 * n, c.stream);
    k_aos_to_soa<<<(unsigned)((6 * n + 255) / 256), 256, 0, c.stream>>>(a->p, n, 6, soa->p);
    LG_LAUNCH();
    auto nx = std::make_shared<DBuf>(3 * n, c.stream);
    auto al = upload_vec(c, std::vector<uint32_t>(alpha, alpha + 6));
    const uint32_t* tw = c.twiddles(logn);
    c.timed("fri_fold", 36.0 * n, 0, [&] {
      k_fold<<<(unsigned)((n / 2 + 255) / 256), 256, 0, c.stream>>>(soa->p, n, al->p, tw, inv(to_mont(2)), nx->p);
      LG_LAUNCH();
    });
    auto aos = std::make_shared<DBuf>(3 * n, c.stream);
    k_soa_to_aos<<<(unsigned)((3 * n + 255) / 256), 256, 0, c.stream>>>(nx->p, n / 2, 6, aos->p);
    LG_LAUNCH();
    from_device(c, out, aos->p, 3 * n, on_device);
  });
}

int lg_grand_product(lg_ctx* ctx, const uint32_t* num, const uint32_t* den, uint64_t n, uint32_t* out, int on_device) {
  return guarded(ctx, [&] {
    Ctx& c = ctx->c;
    if (!num || !den || !out || n == 0) throw Error(LG_ERR_INVALID, "bad arguments");
    auto na = to_device(c, num, 6 * n, on_device), da = to_device(c, den, 6 * n, on_device);
    auto ns = std::make_shared<DBuf>(6 * n, c.stream), ds = std::make_shared<DBuf>(6 * n, c.stream);
    unsigned g6 = (unsigned)((6 * n + 255) / 256), g1 = (unsigned)((n + 255) / 256);
    k_aos_to_soa<<<g6, 256, 0, c.stream>>>(na->p, n, 6, ns->p);
    LG_LAUNCH();
    k_aos_to_soa<<<g6, 256, 0, c.stream>>>(da->p, n, 6, ds->p);
    LG_LAUNCH();
    auto ratio = std::make_shared<DBuf>(6 * n, c.stream);
    k_e6_div_soa<<<g1, 256, 0, c.stream>>>(ns->p, ds->p, n, ratio->p);
    LG_LAUNCH();
    uint32_t nt = (uint32_t)((n + SCAN_TILE - 1) / SCAN_TILE);
    auto totals = std::make_shared<DBuf>(6 * (size_t)nt, c.stream), pre = std::make_shared<DBuf>(6 * (size_t)nt, c.stream);
    auto res = std::make_shared<DBuf>(6 * n, c.stream);
    std::vector<ScanJob> sj = {ScanJob{ratio->p, n, totals->p, pre->p, res->p, nt}};
    auto sd = upload_vec(c, sj);
    k_scan_tiles<<<dim3(nt, 1), SCAN_BLOCK, 0, c.stream>>>((const ScanJob*)sd->p);
    LG_LAUNCH();
    k_tile_prefix<<<1, 64, 0, c.stream>>>((const ScanJob*)sd->p, 1);
    LG_LAUNCH();
    k_gp_finish<<<dim3(g1, 1), 256, 0, c.stream>>>((const ScanJob*)sd->p);
    LG_LAUNCH();
    auto aos = std::make_shared<DBuf>(6 * n, c.stream);
    k_soa_to_aos<<<g6, 256, 0, c.stream>>>(res->p, n, 6, aos->p);
    LG_LAUNCH();
    from_device(c, out, aos->p, 6 * n, on_device);
  });
}

int lg_deep_quotient(lg_ctx* ctx, const uint32_t* lde, uint32_t n_cols, uint64_t rows, const uint32_t alpha[6],
                     const uint32_t z[6], const uint32_t* values, uint32_t* out, int on_device) {
  return guarded(ctx, [&] {
    Ctx& c = ctx->c;
    if (!lde || !alpha || !z || !values || !out || !n_cols || rows < 2 || (rows & (rows - 1)) || rows > (1ull << 24))
      throw Error(LG_ERR_INVALID, "bad arguments");
    int logr = 0;
    while ((1ull << logr) < rows) logr++;
    DBufP src;
    const uint32_t* lanes = lde;
    if (!on_device) {
      src = to_device(c, lde, (size_t)n_cols * rows, 0);
      lanes = src->p;
    }
    E6 a, zz;
    for (int w = 0; w < 6; w++) { a.c[w] = alpha[w]; zz.c[w] = z[w]; }
    // the claimed values are read on the host: bring them back when they live on the device
    std::vector<uint32_t> vals_host;
    if (on_device) {
      vals_host.resize(6 * (size_t)n_cols);
      LG_CK(cudaMemcpyAsync(vals_host.data(), values, vals_host.size() * 4, cudaMemcpyDeviceToHost, c.stream));
      LG_CK(cudaStreamSynchronize(c.stream));
      values = vals_host.data();
    }
    DeepJob jb{};
    std::vector<DeepBundle> bundles;
    E6 run = e6_one(), acc = e6_zero();
    for (uint32_t i = 0; i < n_cols; i++) {
      DeepBundle bu{};
      bu.lane0 = lanes + (size_t)i * rows;
      bu.lane_stride = rows;
      bu.ext = 0;
      bu.mask = 1;
      bu.scale = run;
      E6 v;
      for (int w = 0; w < 6; w++) v.c[w] = values[6 * i + w];
      acc = e6_add(acc, e6_mul(run, v));
      bundles.push_back(bu);
      run = e6_mul(run, a);
    }
    jb.n_points = 1;
    jb.z[0] = zz;
    jb.a[0] = acc;
    auto bd = upload_vec(c, bundles);
    jb.bundles = (const DeepBundle*)bd->p;
    jb.n_bundles = n_cols;
    jb.logn4 = logr;
    jb.tw = c.twiddles(logr);
    auto soa = std::make_shared<DBuf>(6 * rows, c.stream);
    jb.out = soa->p;
    std::vector<DeepJob> jv = {jb};
    auto jd = upload_vec(c, jv);
    c.timed("deep", (4.0 * n_cols + 24.0) * rows, 0, [&] {
      k_deep<<<dim3((unsigned)((rows + 127) / 128), 1), 128, 0, c.stream>>>((const DeepJob*)jd->p);
      LG_LAUNCH();
    });
    auto aos = on_device ? DBufP() : std::make_shared<DBuf>(6 * rows, c.stream);
    uint32_t* dst = on_device ? out : aos->p;
    k_soa_to_aos<<<(unsigned)((6 * rows + 255) / 256), 256, 0, c.stream>>>(soa->p, rows, 6, dst);
    LG_LAUNCH();
    if (!on_device) from_device(c, out, aos->p, 6 * rows, 0);
    else LG_CK(cudaStreamSynchronize(c.stream));
  });
}

int lg_timer_mark(lg_ctx* ctx, uint32_t slot) {
  return guarded(ctx, [&] {
    if (slot >= 16) throw Error(LG_ERR_INVALID, "timer slot must be < 16");
    if (!ctx->c.marks[slot]) LG_CK(cudaEventCreate(&ctx->c.marks[slot]));
    LG_CK(cudaEventRecord(ctx->c.marks[slot], ctx->c.stream));
  });
}

int lg_timer_elapsed(lg_ctx* ctx, uint32_t from, uint32_t to, float* ms) {
  return guarded(ctx, [&] {
    if (from >= 16 || to >= 16 || !ctx->c.marks[from] || !ctx->c.marks[to] || !ms)
      throw Error(LG_ERR_INVALID, "timer slots not recorded");
    LG_CK(cudaEventSynchronize(ctx->c.marks[to]));
    LG_CK(cudaEventElapsedTime(ms, ctx->c.marks[from], ctx->c.marks[to]));
  });
}

uint64_t lg_kernel_launches(void) { return g_launches.load(); }
uint64_t lg_jit_kernels(void) { return xjit_compiled(); }

int lg_profile(lg_ctx* ctx, int enable) {
  return guarded(ctx, [&] {
    LG_CK(cudaStreamSynchronize(ctx->c.stream));
    ctx->c.profiling = enable != 0;
    ctx->c.recs.clear();
    ctx->c.event_next = 0;
  });
}

int lg_profile_report(lg_ctx* ctx, char* buf, size_t* len) {
  return guarded(ctx, [&] {
    if (!len) throw Error(LG_ERR_INVALID, "null length");
    LG_CK(cudaStreamSynchronize(ctx->c.stream));
    struct Acc { uint64_t n = 0; double ms = 0, bytes = 0, perms = 0; };
    std::map<std::string, Acc> acc;
    std::vector<std::map<std::string, Acc>> by_phase(ctx->c.phases.size() + 1);
    for (auto& r : ctx->c.recs) {
      float ms = 0;
      LG_CK(cudaEventElapsedTime(&ms, r.a, r.b));
      for (Acc* a : {&acc[r.name], &by_phase[std::min(r.phase, ctx->c.phases.size())][r.name]}) {
        a->n++;
        a->ms += ms;
        a->bytes += r.bytes;
        a->perms += r.perms;
      }
    }
    std::string js = "{";
    for (auto& kv : acc) {
      char tmp[256];
      snprintf(tmp, sizeof tmp, "%s\"%s\": {\"launches\": %llu, \"ms\": %.6f, \"bytes\": %.0f, \"perms\": %.0f}",
               js.size() > 1 ? ", " : "", kv.first.c_str(), (unsigned long long)kv.second.n, kv.second.ms,
               kv.second.bytes, kv.second.perms);
      js += tmp;
    }
    js += js.size() > 1 ? ", " : "";
    js += "\"phases\": {";
    for (size_t i = 0; i < ctx->c.phases.size(); i++) {
      char tmp[160];
      snprintf(tmp, sizeof tmp, "%s\"%s\": %.4f", i ? ", " : "", ctx->c.phases[i].first.c_str(), ctx->c.phases[i].second);
      js += tmp;
    }
    js += "}, \"kernels_by_phase\": {";
    bool first = true;
    for (size_t i = 0; i < ctx->c.phases.size(); i++) {
      if (by_phase[i].empty()) continue;
      js += first ? "\"" : ", \"";
      first = false;
      js += ctx->c.phases[i].first + "\": {";
      bool f2 = true;
      for (auto& kv : by_phase[i]) {
        char tmp[256];
        snprintf(tmp, sizeof tmp, "%s\"%s\": {\"launches\": %llu, \"ms\": %.6f, \"perms\": %.0f}", f2 ? "" : ", ",
                 kv.first.c_str(), (unsigned long long)kv.second.n, kv.second.ms, kv.second.perms);
        f2 = false;
        js += tmp;
      }
      js += "}";
    }
    // launch timeline on the context's stream: kernel, phase index, start
    // (ms after the first recorded launch began) and duration
    js += "}, \"timeline\": [";
    for (size_t i = 0; i < ctx->c.recs.size(); i++) {
      const auto& r = ctx->c.recs[i];
      float t0 = 0, ms = 0;
      LG_CK(cudaEventElapsedTime(&t0, ctx->c.recs[0].a, r.a));
      LG_CK(cudaEventElapsedTime(&ms, r.a, r.b));
      char tmp[192];
      snprintf(tmp, sizeof tmp, "%s[\"%s\", %llu, %.4f, %.4f]", i ? ", " : "", r.name, (unsigned long long)r.phase, t0, ms);
      js += tmp;
    }
    js += "]}";
    if (!buf || *len < js.size() + 1) {
      *len = js.size() + 1;
      throw Error(LG_ERR_BUFFER, "report buffer too small");
    }
    memcpy(buf, js.c_str(), js.size() + 1);
    *len = js.size() + 1;
  });
}

}  // extern "C"
