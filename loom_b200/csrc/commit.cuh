// PCS commit on the device (internal/fri/commitment.go:259-386): RS/LDE of
// every lane, pair-leaf Poseidon2 hashing, Merkle tree with level injections.
#pragma once
#include <mutex>
#include <type_traits>

#include "host.cuh"
#include "ntt_large.cuh"

namespace lg {

inline DBufP upload_words(Ctx& c, const void* data, size_t bytes) {
  auto b = std::make_shared<DBuf>(std::max<size_t>(1, (bytes + 3) / 4), c.stream);
  if (bytes) c.h2d(b->p, data, bytes);
  return b;
}
template <class T> inline DBufP upload_vec(Ctx& c, const std::vector<T>& v) {
  return upload_words(c, v.data(), v.size() * sizeof(T));
}

// The dynamic shared-memory limit is a property of the kernel function, shared
// by every context and thread in the process: it is only ever raised, so a
// launch of one context never finds it lowered by another.
inline std::mutex g_smem_mu;
inline std::map<const void*, size_t> g_smem_set;
template <class K> inline void allow_smem(K kernel, size_t bytes) {
  std::lock_guard<std::mutex> lk(g_smem_mu);
  size_t& cur = g_smem_set[(const void*)kernel];
  if (bytes <= cur) return;
  LG_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
}

// 16 elements per thread for n >= 16 (radix-16 passes), up to 1024 threads.
// Calls f(std::integral_constant<int, L>{}) with L = logn for the
// shared-memory transform sizes 2^4..2^14 (kernels instantiated per size),
// L = 0 (size read at run time) for the others.
template <class F> inline void with_ntt_size(int logn, F&& f) {
  switch (logn) {
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 5: f(std::integral_constant<int, 5>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 7: f(std::integral_constant<int, 7>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 9: f(std::integral_constant<int, 9>{}); break;
    case 10: f(std::integral_constant<int, 10>{}); break;
    case 11: f(std::integral_constant<int, 11>{}); break;
    case 12: f(std::integral_constant<int, 12>{}); break;
    case 13: f(std::integral_constant<int, 13>{}); break;
    case 14: f(std::integral_constant<int, 14>{}); break;
    default: f(std::integral_constant<int, 0>{}); break;
  }
}
inline int ntt_threads(int logn) { return logn < 4 ? 32 : std::max(32, std::min(1024, 1 << (logn - 4))); }
// shared words of one pad16 array of n = 2^logn points
inline size_t pad16_words(int logn) { return ((size_t)1 << logn) + ((size_t)1 << logn) / 16 + 1; }

constexpr int MAX_NTT_LOG = 22;  // the largest loom module, 2^22 rows
inline void check_ntt_size(int logn) {
  if (logn > MAX_NTT_LOG) throw Error(LG_ERR_UNSUPPORTED, "transforms above 2^22 points are not supported");
}

// Runs four-step transforms of 2^logn points (logn > SMEM_NTT_MAX_LOG), all
// jobs of one direction, in chunks whose scratch stays below 256 MiB.
inline void big_ntt(Ctx& c, std::vector<BigNtt> jobs, int logn, bool inverse, const char* tag, double bytes_per_job) {
  if (jobs.empty()) return;
  const int logr = logn / 2, logc = logn - logr;
  if (logr < 7 || logc > 11) throw Error(LG_ERR_UNSUPPORTED, "four-step transform size out of range");
  const size_t n = (size_t)1 << logn;
  const uint32_t* tw_c = c.twiddles16(logc);
  const uint32_t* tw_r = c.twiddles16(logr);
  // the large roots' powers as two small tables each (mul_split): w_n and,
  // for the coset shifts, w_{4n}
  const uint2* tw_n = c.split_powers(logn);
  const uint2* t2s = c.split_powers(logn + RATE_LOG);
  for (auto& j : jobs) {
    if (j.t2 && j.m2_mask != (uint32_t)((n << RATE_LOG) - 1))
      throw Error(LG_ERR_INVALID, "four-step coset table of another size");
    j.c0c = from_mont(j.c0);
    j.c0s = shoup(j.c0c);
  }
  // scratch chunks of 2^26 words at most (256 MiB)
  const size_t per = std::max<size_t>(1, ((size_t)1 << 26) / n);
  const size_t smem_a = tile_words(logc) * 4, smem_b = tile_words(logr) * 4;
  const unsigned thr_a = (unsigned)std::min<size_t>(512, (size_t)1 << logc);
  const unsigned thr_b = (unsigned)std::min<size_t>(512, (size_t)1 << logr);
  for (size_t first = 0; first < jobs.size(); first += per) {
    size_t cnt = std::min(per, jobs.size() - first);
    auto scratch = std::make_shared<DBuf>(cnt * n, c.stream);
    std::vector<BigNtt> v(jobs.begin() + first, jobs.begin() + first + cnt);
    for (size_t i = 0; i < cnt; i++) v[i].scratch = scratch->p + i * n;
    auto jd = upload_vec(c, v);
    c.timed(tag, bytes_per_job * cnt, 0, [&] {
      with_tile_size(logc, [&](auto LC) {
        constexpr int C_ = decltype(LC)::value;
        allow_smem(k_big_pass_a<C_>, smem_a);
        k_big_pass_a<C_><<<dim3((1u << logr) / BIG_TILE, (unsigned)cnt), thr_a, smem_a, c.stream>>>(
            (const BigNtt*)jd->p, logn, logr, inverse ? 1 : 0, tw_n, t2s, tw_c);
        LG_LAUNCH();
      });
      with_tile_size(logr, [&](auto LR) {
        constexpr int R_ = decltype(LR)::value;
        allow_smem(k_big_pass_b<R_>, smem_b);
        k_big_pass_b<R_><<<dim3((1u << logc) / BIG_TILE, (unsigned)cnt), thr_b, smem_b, c.stream>>>(
            (const BigNtt*)jd->p, logc, inverse ? 1 : 0, tw_r);
        LG_LAUNCH();
      });
    });
  }
}

inline BigNtt big_job(const uint32_t* in, uint32_t* out, uint32_t c0, bool bitrev_out) {
  BigNtt j{};
  j.in = in;
  j.out = out;
  j.c0 = c0;
  j.out_bitrev = bitrev_out ? 1 : 0;
  return j;
}

// One k_lde launch over lanes that share a size (four-step transforms above
// 2^14 points).
inline void launch_lde(Ctx& c, const std::vector<LdeLane>& lanes, uint32_t log_n, bool from_coeffs) {
  if (lanes.empty()) return;
  check_ntt_size((int)log_n);
  size_t n = (size_t)1 << log_n;
  if ((int)log_n > SMEM_NTT_MAX_LOG) {
    DBufP tmp;
    std::vector<const uint32_t*> coef(lanes.size());
    std::vector<BigNtt> inv_jobs, fwd_jobs;
    bool need_tmp = false;
    for (auto& L : lanes) need_tmp |= !from_coeffs && !L.coef;
    if (need_tmp) tmp = std::make_shared<DBuf>(lanes.size() * n, c.stream);
    for (size_t i = 0; i < lanes.size(); i++) {
      if (from_coeffs) {
        coef[i] = lanes[i].src;
        if (lanes[i].coef)
          LG_CK(cudaMemcpyAsync(lanes[i].coef, lanes[i].src, n * 4, cudaMemcpyDeviceToDevice, c.stream));
      } else {
        uint32_t* dst = lanes[i].coef ? lanes[i].coef : tmp->p + i * n;
        inv_jobs.push_back(big_job(lanes[i].src, dst, inv(to_mont((uint32_t)n)), false));
        coef[i] = dst;
      }
    }
    big_ntt(c, inv_jobs, (int)log_n, true, "lde", 8.0 * n);
    const uint32_t* tw4 = c.twiddles((int)log_n + RATE_LOG);
    for (size_t i = 0; i < lanes.size(); i++)
      for (int a = 0; a < (1 << RATE_LOG); a++) {
        BigNtt j = big_job(coef[i], lanes[i].out + (size_t)a * n, MONT_ONE, true);
        j.t2 = tw4;
        j.m2_mask = (uint32_t)((n << RATE_LOG) - 1);
        j.e2 = bitrev32((uint32_t)a, RATE_LOG);
        fwd_jobs.push_back(j);
      }
    big_ntt(c, fwd_jobs, (int)log_n, false, "lde", 20.0 * n / (1 << RATE_LOG));
    return;
  }
  const uint32_t* twn = c.ntt_twiddles((int)log_n);
  const uint32_t* tw4 = c.twiddles((int)log_n + RATE_LOG);
  const size_t smem = 2 * pad16_words((int)log_n) * 4;
  const double bytes = 20.0 * n * lanes.size();
  if (!c.tune.lde_split || log_n < 4) {
    // one block per lane: inverse transform and the coset transforms
    auto tab = upload_vec(c, lanes);
    with_ntt_size((int)log_n, [&](auto L) {
      allow_smem(k_lde<decltype(L)::value>, smem);
      c.timed("lde", bytes, 0, [&] {
        k_lde<decltype(L)::value><<<(unsigned)lanes.size(), ntt_threads((int)log_n), smem, c.stream>>>(
            (const LdeLane*)tab->p, (int)log_n, from_coeffs ? 1 : 0, twn, tw4, inv(to_mont((uint32_t)n)));
        LG_LAUNCH();
      });
    });
    return;
  }
  // split: the inverse transforms (coset 0 and the coefficients) in one
  // launch, then the coset transforms, one block per (lane, coset)
  std::vector<LdeLane> lv = lanes;
  DBufP tmp;
  size_t missing = 0;
  for (auto& L : lv) missing += !from_coeffs && !L.coef;
  if (missing) tmp = std::make_shared<DBuf>(missing * n, c.stream);
  for (size_t i = 0, k = 0; i < lv.size(); i++)
    if (!from_coeffs && !lv[i].coef) lv[i].coef = tmp->p + (k++) * n;
  auto tab = upload_vec(c, lv);
  if (from_coeffs)  // the coefficients themselves are kept when asked for
    for (auto& L : lv)
      if (L.coef) LG_CK(cudaMemcpyAsync(L.coef, L.src, n * 4, cudaMemcpyDeviceToDevice, c.stream));
  with_ntt_size((int)log_n, [&](auto L) {
    constexpr int LG = decltype(L)::value;
    const size_t fsmem = pad16_words((int)log_n) * 4;
    const unsigned thr = (unsigned)std::min<int>(ntt_threads((int)log_n), (int)c.tune.lde_fwd_threads);
    if (!from_coeffs) {
      auto go_inv = [&](auto kern) {
        allow_smem(kern, fsmem);
        c.timed("lde_inv", 8.0 * n * lv.size(), 0, [&] {
          kern<<<(unsigned)lv.size(), thr, fsmem, c.stream>>>((const LdeLane*)tab->p, twn, inv(to_mont((uint32_t)n)));
          LG_LAUNCH();
        });
      };
      if constexpr (LG >= 4) {
        if (thr <= 256) go_inv(k_lde_inv<LG, 256>);
        else if (thr <= 512) go_inv(k_lde_inv<LG, 512>);
        else go_inv(k_lde_inv<LG, 1024>);
      }
    }
    const int first = from_coeffs ? 0 : 1;
    auto go = [&](auto kern) {
      allow_smem(kern, fsmem);
      c.timed("lde", bytes - (from_coeffs ? 0.0 : 8.0 * n * lv.size()), 0, [&] {
        for (size_t l0 = 0; l0 < lv.size(); l0 += 65535) {  // grid y: lanes, at most 65535 a launch
          const dim3 grid((unsigned)((1 << RATE_LOG) - first), (unsigned)std::min<size_t>(65535, lv.size() - l0));
          kern<<<grid, thr, fsmem, c.stream>>>((const LdeLane*)tab->p, (uint32_t)l0, first, twn, tw4);
          LG_LAUNCH();
        }
      });
    };
    if constexpr (LG >= 4) {
      if (thr <= 256) go(k_lde_fwd<LG, 256>);
      else if (thr <= 512) go(k_lde_fwd<LG, 512>);
      else go(k_lde_fwd<LG, 1024>);
    }
  });
}

// Poseidon2 lane mapping for a launch of `parallel` independent permutation
// chains (leaves, nodes of one level): with at least `per_sm` of them per SM,
// one thread per chain (fewest instructions per permutation); otherwise six
// lanes per chain for a dependent chain six times shorter.  Measured on B200:
// one thread per chain wins for leaf hashing and injection chains from 128
// chains per SM, for one-permutation Merkle levels from 512 (Ctx::tune).
inline bool p2_per_thread(const Ctx& c, uint64_t parallel, uint32_t per_sm) {
  return c.leaf_mapping == 1 || (c.leaf_mapping == 0 && parallel >= (uint64_t)c.sm_count * per_sm);
}

inline void launch_leaves(Ctx& c, const std::vector<LeafGroup>& gs) {
  if (gs.empty()) return;
  uint32_t max_leaves = 0;
  double bytes = 0, perms = 0;
  for (auto& g : gs) {
    max_leaves = std::max(max_leaves, g.n_leaves);
    uint32_t total = 3 + 2 * g.nb + 12 * g.ne;
    bytes += 8.0 * g.n_leaves * (g.nb + 6 * g.ne) + 32.0 * g.n_leaves;
    perms += (double)g.n_leaves * ((total + 15) / 16);
  }
  auto tab = upload_vec(c, gs);
  uint64_t all_leaves = 0;
  for (auto& g : gs) all_leaves += g.n_leaves;
  bool per_thread = p2_per_thread(c, all_leaves, c.tune.p2_leaf_min_per_sm);
  const unsigned lb = c.tune.leaf_block;
  c.timed("hash_leaves", bytes, perms, [&] {
    if (per_thread)
      k_hash_leaves1<<<dim3((max_leaves + lb - 1) / lb, (unsigned)gs.size()), lb, 0, c.stream>>>((const LeafGroup*)tab->p);
    else
      k_hash_leaves<<<dim3((max_leaves + 19) / 20, (unsigned)gs.size()), 128, 0, c.stream>>>((const LeafGroup*)tab->p);
    LG_LAUNCH();
  });
}

inline LeafGroup leaf_group(const uint32_t* lde, uint32_t nb, uint32_t ne, uint32_t log_rows, uint32_t* out) {
  LeafGroup g;
  uint64_t rows = 1ull << log_rows;
  g.base = lde;
  g.ext = lde + (uint64_t)nb * rows;
  g.stride = rows;
  g.nb = nb;
  g.ne = ne;
  g.n_leaves = (uint32_t)(rows / 2);
  g.out = out;
  return g;
}

struct LdeOut {
  DBufP lde;   // lanes x 4n
  DBufP coef;  // lanes x n (optional)
  uint32_t lanes = 0, log_n = 0;
};

// LDE of `src` lanes (all of 2^log_n rows) into one buffer (used by lg_rs_encode).
inline LdeOut lde_lanes(Ctx& c, const std::vector<const uint32_t*>& src, uint32_t log_n, bool from_coeffs,
                        bool keep_coef) {
  check_ntt_size((int)log_n);
  LdeOut r;
  r.lanes = (uint32_t)src.size();
  r.log_n = log_n;
  size_t n = (size_t)1 << log_n;
  r.lde = std::make_shared<DBuf>(src.size() * (n << RATE_LOG), c.stream);
  if (keep_coef) r.coef = std::make_shared<DBuf>(src.size() * n, c.stream);
  std::vector<LdeLane> lanes;
  for (size_t i = 0; i < src.size(); i++)
    lanes.push_back(LdeLane{src[i], r.lde->p + i * (n << RATE_LOG), keep_coef ? r.coef->p + i * n : nullptr});
  launch_lde(c, lanes, log_n, from_coeffs);
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

// Levels below merkle_tail run in one block (k_merkle_tail); above it, a
// launch per merkle_subtree input nodes builds one subtree per block (or a
// launch per level).  Six lanes per permutation, five permutations per warp,
// sized for the widest level of a block.
inline unsigned tail_threads(uint32_t top, int fold_first) {
  uint32_t perms = std::max(1u, fold_first ? top : top / 2);
  return std::min(1024u, (perms + 4) / 5 * 32);
}

// nodes must already hold the leaves at [n_leaves, 2 n_leaves).  Reads the
// root back (the transcript needs it) unless read_root is false.
// With fs, a tree whose top runs as one k_merkle_tail block also gets the
// challenge over its root there (fs->out); returns whether it did (else the
// caller computes it).
inline bool build_tree(Ctx& c, TreeDev& t, bool read_root = true, const FsTail* fs = nullptr) {
  const uint32_t nl = 1u << t.log_leaves;
  for (size_t k = 0; k < t.inj.size(); k++)
    if (t.inj_log_w[k] > t.log_leaves || (k && t.inj_log_w[k] > t.inj_log_w[k - 1]))
      throw Error(LG_ERR_INVALID, "injection widths must not increase");
  std::vector<const uint32_t*> ip;
  std::vector<uint32_t> sh;
  std::vector<InjRef> refs;
  for (size_t k = 0; k < t.inj.size(); k++) {
    ip.push_back(t.inj[k]->p);
    sh.push_back(t.log_leaves - t.inj_log_w[k]);
    refs.push_back(InjRef{t.inj[k]->p, 1u << t.inj_log_w[k]});
  }
  t.inj_ptrs = upload_vec(c, ip);
  t.inj_shift = upload_vec(c, sh);
  auto ref_tab = upload_vec(c, refs);
  size_t next = 0;
  auto fold = [&](uint32_t start) {
    size_t first = next;
    while (next < t.inj.size() && (1u << t.inj_log_w[next]) == start) next++;
    if (next == first) return;
    const uint32_t* const* tab = (const uint32_t* const*)t.inj_ptrs->p + first;
    uint32_t cnt = (uint32_t)(next - first);
    c.timed("merkle_inject", 96.0 * start * cnt, (double)start * cnt, [&] {
      if (p2_per_thread(c, start, c.tune.p2_inject_min_per_sm)) {
        // small blocks (one warp by default): chains are few (down to ~200
        // per SM) and long, so small blocks spread them evenly over the SMs
        const unsigned ib = c.tune.inject_block;
        k_merkle_inject1<<<(start + ib - 1) / ib, ib, 0, c.stream>>>(t.nodes->p, start, tab, cnt);
      } else
        k_merkle_inject<<<(start + 19) / 20, 128, 0, c.stream>>>(t.nodes->p, start, tab, cnt);
      LG_LAUNCH();
    });
  };
  auto level = [&](uint32_t start) {
    c.timed("merkle_level", 96.0 * start, (double)start, [&] {
      if (p2_per_thread(c, start, c.tune.p2_node_min_per_sm))
        k_merkle_level1<<<(start + 127) / 128, 128, 0, c.stream>>>(t.nodes->p, start);
      else
        k_merkle_level<<<(start + 19) / 20, 128, 0, c.stream>>>(t.nodes->p, start);
      LG_LAUNCH();
    });
  };
  bool fused = false;
  // blocks = 1: the tree top from width `top` (k_merkle_tail); blocks > 1:
  // the levels top/2 .. blocks, one subtree per block
  auto subtrees = [&](uint32_t top, int fold_first, uint32_t blocks) {
    double perms = (double)(top - blocks);  // nodes of the levels built, plus their injections
    for (size_t k = 0; k < t.inj.size(); k++) {
      const uint32_t w = 1u << t.inj_log_w[k];
      if ((w < top && w >= blocks) || (fold_first && w == top)) perms += w;
    }
    const bool with_fs = blocks == 1 && fs;
    if (with_fs) fused = true;
    c.timed(blocks == 1 ? "merkle_tail" : "merkle_level", 96.0 * perms, perms, [&] {
      // at least one warp: the challenge needs one
      const unsigned thr = std::max(32u, tail_threads(top / blocks, fold_first));
      k_merkle_tail<<<blocks, thr, 0, c.stream>>>(t.nodes->p, top, fold_first, (const InjRef*)ref_tab->p,
                                                  (uint32_t)refs.size(), with_fs ? *fs : FsTail{});
      LG_LAUNCH();
    });
  };
  const uint32_t tail_w = c.tune.merkle_tail, sub = c.tune.merkle_subtree;
  // a block chains at most 64 injections of one width
  bool chain_ok = true;
  for (size_t k = 0; k < t.inj.size(); k++) {
    size_t same = 0;
    for (size_t q = 0; q < t.inj.size(); q++) same += t.inj_log_w[q] == t.inj_log_w[k];
    if ((1u << t.inj_log_w[k]) < nl && same > 64) chain_ok = false;
  }
  if (!c.batched || !chain_ok) {
    fold(nl);
    for (uint32_t start = nl >> 1; start >= 1; start >>= 1) { level(start); fold(start); }
  } else if (nl <= tail_w) {
    subtrees(nl, 1, 1);
  } else {
    fold(nl);
    uint32_t start = nl;
    while (start > tail_w) {
      // one launch reaches down to `stop`: start / sub at most, and not
      // through a level with injections above the tail, whose chains run
      // GPU-wide (fold) rather than on a block's few warps
      const uint32_t lo = sub >= 2 ? std::max(tail_w, start / sub) : start;
      uint32_t stop = lo;
      for (size_t k = 0; k < t.inj.size(); k++) {
        const uint32_t w = 1u << t.inj_log_w[k];
        if (w >= lo && w < start) stop = std::max(stop, 2 * w);
      }
      if (stop < start) {
        subtrees(start, 0, stop);
        start = stop;
      } else {
        level(start >> 1);
        fold(start >> 1);
        start >>= 1;
      }
    }
    subtrees(start, 0, 1);
  }
  if (!read_root) return fused;  // the root stays on the device (nodes[1])
  uint32_t* h = c.host_staging(8);
  c.d2h(h, t.nodes->p + 8, 8);
  memcpy(t.root.v, h, 32);
  return fused;
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
// read_root = false leaves the root on the device (tree.nodes[1]), unread.
inline Committed commit(Ctx& c, const std::vector<GroupSpec>& gs, bool keep_coef, bool read_root = true) {
  if (gs.empty()) throw Error(LG_ERR_INVALID, "commit: empty batch");
  Committed cm;
  for (size_t i = 0; i < gs.size(); i++) {
    if (gs[i].lanes.size() != gs[i].nb + 6 * (size_t)gs[i].ne) throw Error(LG_ERR_INVALID, "commit: lane count");
    if (gs[i].lanes.empty()) throw Error(LG_ERR_INVALID, "commit: group has no polynomials");
    check_ntt_size((int)gs[i].log_n);
    cm.order.push_back((int)i);
  }
  std::stable_sort(cm.order.begin(), cm.order.end(), [&](int a, int b) { return gs[a].log_n > gs[b].log_n; });
  // LDE buffers, one per group, slices of one allocation
  std::map<uint32_t, std::vector<LdeLane>> by_size;
  std::vector<std::vector<LdeLane>> per_group(gs.size());
  size_t lde_words = 0, coef_words = 0;
  for (auto& g : gs) {
    lde_words += g.lanes.size() * ((size_t)1 << (g.log_n + RATE_LOG));
    coef_words += g.lanes.size() * ((size_t)1 << g.log_n);
  }
  auto lde_all = std::make_shared<DBuf>(lde_words, c.stream);
  auto coef_all = keep_coef ? std::make_shared<DBuf>(coef_words, c.stream) : DBufP();
  size_t lde_off = 0, coef_off = 0;
  for (size_t i = 0; i < gs.size(); i++) {
    LdeOut o;
    o.lanes = (uint32_t)gs[i].lanes.size();
    o.log_n = gs[i].log_n;
    size_t n = (size_t)1 << o.log_n;
    o.lde = dbuf_slice(lde_all, lde_off, o.lanes * (n << RATE_LOG));
    lde_off += o.lanes * (n << RATE_LOG);
    if (keep_coef) {
      o.coef = dbuf_slice(coef_all, coef_off, o.lanes * n);
      coef_off += o.lanes * n;
    }
    for (uint32_t l = 0; l < o.lanes; l++) {
      LdeLane L{gs[i].lanes[l], o.lde->p + l * (n << RATE_LOG), keep_coef ? o.coef->p + l * n : nullptr};
      (c.batched ? by_size[o.log_n] : per_group[i]).push_back(L);
    }
    cm.groups.push_back(o);
  }
  // the from_coeffs flag is per batch: all groups of a commit share it
  for (size_t i = 1; i < gs.size(); i++)
    if (gs[i].from_coeffs != gs[0].from_coeffs) throw Error(LG_ERR_INVALID, "commit: mixed input forms");
  if (c.batched) for (auto& kv : by_size) launch_lde(c, kv.second, kv.first, gs[0].from_coeffs);
  else for (size_t i = 0; i < gs.size(); i++) launch_lde(c, per_group[i], gs[i].log_n, gs[i].from_coeffs);
  // leaves: the largest group fills the tree's leaf level, the others are injections
  const GroupSpec& top = gs[cm.order[0]];
  TreeDev& t = cm.tree;
  t.log_leaves = top.log_n + RATE_LOG - 1;
  t.nodes = std::make_shared<DBuf>((size_t)16 << t.log_leaves, c.stream);
  std::vector<LeafGroup> lg;
  for (size_t k = 0; k < cm.order.size(); k++) {
    int gi = cm.order[k];
    uint32_t log_rows = gs[gi].log_n + RATE_LOG;
    uint32_t* out;
    if (k == 0) out = t.nodes->p + ((size_t)8 << t.log_leaves);
    else {
      auto lv = std::make_shared<DBuf>((size_t)8 << (log_rows - 1), c.stream);
      t.inj.push_back(lv);
      t.inj_log_w.push_back(log_rows - 1);
      out = lv->p;
    }
    lg.push_back(leaf_group(cm.groups[gi].lde->p, gs[gi].nb, gs[gi].ne, log_rows, out));
  }
  if (c.batched) launch_leaves(c, lg);
  else for (auto& g : lg) launch_leaves(c, {g});
  build_tree(c, t, read_root);
  return cm;
}

}  // namespace lg
