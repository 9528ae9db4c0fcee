// PCS commit on the device (internal/fri/commitment.go:259-386): RS/LDE of
// every lane, pair-leaf Poseidon2 hashing, Merkle tree with level injections.
#pragma once
#include "host.cuh"

namespace lg {

// Device array of lane pointers, uploaded from a host vector.
inline DBufP upload_ptrs(Ctx& c, const std::vector<const uint32_t*>& v) {
  auto b = std::make_shared<DBuf>(std::max<size_t>(2, v.size() * 2), c.stream);
  if (!v.empty()) c.h2d(b->p, v.data(), v.size() * sizeof(void*));
  return b;
}
inline DBufP upload_words(Ctx& c, const void* data, size_t bytes) {
  auto b = std::make_shared<DBuf>(std::max<size_t>(1, (bytes + 3) / 4), c.stream);
  if (bytes) c.h2d(b->p, data, bytes);
  return b;
}

// k_lde_small / k_coset_eval variants that take a table of lane pointers.
__global__ void k_lde_ptrs(const uint32_t* const* src, int logn, int from_coeffs, const uint32_t* tw_n,
                           const uint32_t* tw_4n, uint32_t n_inv, uint32_t* out, uint32_t* coef) {
  extern __shared__ uint32_t sm[];
  const uint32_t n = 1u << logn;
  uint32_t* A = sm;
  uint32_t* B = sm + n;
  const uint32_t* s = src[blockIdx.x];
  if (from_coeffs) {
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) A[k] = s[k];
    __syncthreads();
  } else {
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) A[bitrev32(k, logn)] = s[k];
    __syncthreads();
    smem_dit(A, logn, tw_n, true);
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) A[k] = mul(A[k], n_inv);
    __syncthreads();
  }
  if (coef) {
    uint32_t* cf = coef + (uint64_t)blockIdx.x * n;
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) cf[k] = A[k];
  }
  uint32_t* o = out + (uint64_t)blockIdx.x * ((uint64_t)n << RATE_LOG);
  const uint32_t big = n << RATE_LOG;
  for (int a = 0; a < (1 << RATE_LOG); a++) {
    const uint32_t e = bitrev32((uint32_t)a, RATE_LOG);
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) B[k] = mul(A[k], __ldg(tw_4n + ((e * k) & (big - 1))));
    __syncthreads();
    smem_dif(B, logn, tw_n, false);
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) o[(uint64_t)a * n + k] = B[k];
    __syncthreads();
  }
}

__global__ void k_coset_eval_ptrs(const uint32_t* const* coef, int logn, const uint32_t* tw_n, const uint32_t* tw_4n,
                                  const uint32_t* gpow, uint32_t* out) {
  extern __shared__ uint32_t sm[];
  const uint32_t n = 1u << logn, lane = blockIdx.x, c = blockIdx.y;
  const uint32_t* s = coef[lane];
  const uint32_t big = n << RATE_LOG;
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x)
    sm[k] = mul(mul(s[k], __ldg(gpow + k)), __ldg(tw_4n + ((c * k) & (big - 1))));
  __syncthreads();
  smem_dif(sm, logn, tw_n, false);
  uint32_t* o = out + (uint64_t)lane * big + (uint64_t)c * n;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) o[j] = sm[bitrev32(j, logn)];
}

template <class K> inline void allow_smem(K kernel, size_t bytes) {
  LG_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

inline int ntt_threads(int logn) { return std::max(32, std::min(512, 1 << std::max(0, logn - 1))); }

inline void check_ntt_size(int logn) {
  if (logn > SMEM_NTT_MAX_LOG)
    throw Error(LG_ERR_UNSUPPORTED, "module sizes above 2^" + std::to_string(SMEM_NTT_MAX_LOG) +
                                        " rows are not supported by this build");
}

struct LdeOut {
  DBufP lde;   // lanes x 4n
  DBufP coef;  // lanes x n (optional)
  uint32_t lanes = 0, log_n = 0;
};

inline LdeOut lde_lanes(Ctx& c, const std::vector<const uint32_t*>& src, uint32_t log_n, bool from_coeffs,
                        bool keep_coef) {
  check_ntt_size((int)log_n);
  LdeOut r;
  r.lanes = (uint32_t)src.size();
  r.log_n = log_n;
  size_t n = (size_t)1 << log_n;
  r.lde = std::make_shared<DBuf>(src.size() * (n << RATE_LOG), c.stream);
  if (keep_coef) r.coef = std::make_shared<DBuf>(src.size() * n, c.stream);
  if (src.empty()) return r;
  auto ptrs = upload_ptrs(c, src);
  const uint32_t* twn = c.twiddles((int)log_n);
  const uint32_t* tw4 = c.twiddles((int)log_n + RATE_LOG);
  size_t smem = 2 * n * 4;
  allow_smem(k_lde_ptrs, smem);
  c.timed("lde", 20.0 * n * src.size(), 0, [&] {
    k_lde_ptrs<<<(unsigned)src.size(), ntt_threads((int)log_n), smem, c.stream>>>(
        (const uint32_t* const*)ptrs->p, (int)log_n, from_coeffs ? 1 : 0, twn, tw4, inv(to_mont((uint32_t)n)),
        r.lde->p, keep_coef ? r.coef->p : nullptr);
    LG_LAUNCH();
  });
  return r;
}

// ---------------------------------------------------------------- trees
struct TreeDev {
  DBufP nodes;                        // 2 * n_leaves digests, 1-indexed
  uint32_t log_leaves = 0;
  std::vector<DBufP> inj;             // injection leaves in schedule order
  std::vector<uint32_t> inj_log_w;
  DBufP inj_ptrs, inj_shift;          // device tables for path gathers
  Digest root;
};

// nodes must already hold the leaves at [n_leaves, 2 n_leaves).
inline void build_tree(Ctx& c, TreeDev& t) {
  const uint32_t nl = 1u << t.log_leaves;
  size_t next = 0;
  auto fold = [&](uint32_t start) {
    std::vector<const uint32_t*> ptrs;
    while (next < t.inj.size() && (1u << t.inj_log_w[next]) == start) ptrs.push_back(t.inj[next++]->p);
    if (ptrs.empty()) return;
    auto tab = upload_ptrs(c, ptrs);
    c.timed("merkle_inject", 96.0 * start * ptrs.size(), (double)start * ptrs.size(), [&] {
      k_merkle_inject<<<(start + 127) / 128, 128, 0, c.stream>>>(t.nodes->p, start, (const uint32_t* const*)tab->p,
                                                                  (uint32_t)ptrs.size());
      LG_LAUNCH();
    });
  };
  for (size_t k = 0; k < t.inj.size(); k++)
    if (t.inj_log_w[k] > t.log_leaves || (k && t.inj_log_w[k] > t.inj_log_w[k - 1]))
      throw Error(LG_ERR_INVALID, "injection widths must not increase");
  fold(nl);
  for (uint32_t start = nl >> 1; start >= 1; start >>= 1) {
    c.timed("merkle_level", 96.0 * start, (double)start, [&] {
      k_merkle_level<<<(start + 127) / 128, 128, 0, c.stream>>>(t.nodes->p, start);
      LG_LAUNCH();
    });
    fold(start);
  }
  std::vector<const uint32_t*> ip;
  std::vector<uint32_t> sh;
  for (size_t k = 0; k < t.inj.size(); k++) { ip.push_back(t.inj[k]->p); sh.push_back(t.log_leaves - t.inj_log_w[k]); }
  t.inj_ptrs = upload_ptrs(c, ip);
  t.inj_shift = upload_words(c, sh.data(), sh.size() * 4);
  uint32_t* h = c.host_staging(8);
  c.d2h(h, t.nodes->p + 8, 8);
  memcpy(t.root.v, h, 32);
}

inline void hash_leaves(Ctx& c, const uint32_t* lde, uint32_t nb, uint32_t ne, uint32_t log_rows, uint32_t* out) {
  LeafGroup g;
  uint64_t rows = 1ull << log_rows;
  g.base = lde;
  g.ext = lde + (uint64_t)nb * rows;
  g.stride = rows;
  g.nb = nb;
  g.ne = ne;
  g.n_leaves = (uint32_t)(rows / 2);
  g.out = out;
  uint32_t total = 3 + 2 * nb + 12 * ne;
  c.timed("hash_leaves", 4.0 * rows * (nb + 6 * ne) + 32.0 * g.n_leaves, (double)g.n_leaves * ((total + 15) / 16), [&] {
    k_hash_leaves<<<(g.n_leaves + 127) / 128, 128, 0, c.stream>>>(g);
    LG_LAUNCH();
  });
}

struct GroupSpec {
  uint32_t log_n;                       // Lagrange rows
  std::vector<const uint32_t*> lanes;   // nb base lanes, then 6 lanes per ext column
  uint32_t nb, ne;
  bool from_coeffs;
};
struct Committed {
  std::vector<int> order;               // sorted position -> declaration index
  std::vector<LdeOut> groups;           // declaration order
  TreeDev tree;
};

// RSCommit.Commit: groups sorted by size (stable, descending); the largest
// is the leaf level, the others fold in as level injections.
inline Committed commit(Ctx& c, const std::vector<GroupSpec>& gs, bool keep_coef) {
  if (gs.empty()) throw Error(LG_ERR_INVALID, "commit: empty batch");
  Committed cm;
  for (size_t i = 0; i < gs.size(); i++) {
    if (gs[i].lanes.size() != gs[i].nb + 6 * (size_t)gs[i].ne) throw Error(LG_ERR_INVALID, "commit: lane count");
    if (gs[i].lanes.empty()) throw Error(LG_ERR_INVALID, "commit: group has no polynomials");
    cm.order.push_back((int)i);
  }
  std::stable_sort(cm.order.begin(), cm.order.end(), [&](int a, int b) { return gs[a].log_n > gs[b].log_n; });
  for (auto& g : gs) cm.groups.push_back(lde_lanes(c, g.lanes, g.log_n, g.from_coeffs, keep_coef));
  const GroupSpec& top = gs[cm.order[0]];
  TreeDev& t = cm.tree;
  t.log_leaves = top.log_n + RATE_LOG - 1;
  t.nodes = std::make_shared<DBuf>((size_t)16 << t.log_leaves, c.stream);
  for (size_t k = 0; k < cm.order.size(); k++) {
    int gi = cm.order[k];
    const LdeOut& l = cm.groups[gi];
    uint32_t log_rows = gs[gi].log_n + RATE_LOG;
    if (k == 0) {
      hash_leaves(c, l.lde->p, gs[gi].nb, gs[gi].ne, log_rows, t.nodes->p + ((size_t)8 << t.log_leaves));
    } else {
      auto lv = std::make_shared<DBuf>((size_t)8 << (log_rows - 1), c.stream);
      hash_leaves(c, l.lde->p, gs[gi].nb, gs[gi].ne, log_rows, lv->p);
      t.inj.push_back(lv);
      t.inj_log_w.push_back(log_rows - 1);
    }
  }
  build_tree(c, t);
  return cm;
}

}  // namespace lg
