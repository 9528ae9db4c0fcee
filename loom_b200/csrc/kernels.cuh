// sm_100a kernels of the Poseidon2 prove path.  All field data is Montgomery
// words; an E6 column is stored as 6 base "lanes" (structure of arrays), so
// every transform and gather works on plain u32 columns.
#pragma once
#include <cuda_runtime.h>

#include "field.cuh"
#include "p2_coop.cuh"
#include "ntt16.cuh"

namespace lg {

constexpr int RATE_LOG = 2;  // blowup 4 (internal/constants/const.go:24)
constexpr int SMEM_NTT_MAX_LOG = 14;
constexpr uint32_t LEAF_TAG = 0x4c454146u, NODE_TAG = 0x4e4f4445u;

// ---------------------------------------------------------------- twiddles
// tw[j] = w_n^j for j < n, w_n = root_of_unity(log n).
__global__ void k_fill_powers(uint32_t* out, uint64_t n, uint32_t base, uint32_t start) {
  uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j < n) out[j] = mul(start, mont_pow(base, j));
}

// ---------------------------------------------------------------- smem NTT
// Radix-2 stages over a block-resident array A of n = 2^logn words.
// tw: table of w_n^j (j < n) for this n; `inverse` uses w_n^-j = w_n^(n-j).
__device__ __forceinline__ uint32_t tw_at(const uint32_t* tw, uint32_t idx, uint32_t mask, bool inverse) {
  return inverse ? __ldg(tw + ((0u - idx) & mask)) : __ldg(tw + idx);
}

// DIT: bit-reversed input, natural output.
__device__ void smem_dit(uint32_t* A, int logn, const uint32_t* tw, bool inverse) {
  const uint32_t n = 1u << logn, mask = n - 1;
  for (int s = 1; s <= logn; s++) {
    const uint32_t half = 1u << (s - 1);
    for (uint32_t t = threadIdx.x; t < n / 2; t += blockDim.x) {
      uint32_t j = t & (half - 1);
      uint32_t i0 = ((t >> (s - 1)) << s) | j, i1 = i0 + half;
      uint32_t w = tw_at(tw, j << (logn - s), mask, inverse);
      uint32_t u = A[i0], v = mul(A[i1], w);
      A[i0] = add(u, v);
      A[i1] = sub(u, v);
    }
    __syncthreads();
  }
}

// DIF: natural input, bit-reversed output.
__device__ void smem_dif(uint32_t* A, int logn, const uint32_t* tw, bool inverse) {
  const uint32_t n = 1u << logn, mask = n - 1;
  for (int s = logn; s >= 1; s--) {
    const uint32_t half = 1u << (s - 1);
    for (uint32_t t = threadIdx.x; t < n / 2; t += blockDim.x) {
      uint32_t j = t & (half - 1);
      uint32_t i0 = ((t >> (s - 1)) << s) | j, i1 = i0 + half;
      uint32_t w = tw_at(tw, j << (logn - s), mask, inverse);
      uint32_t u = A[i0], v = A[i1];
      A[i0] = add(u, v);
      A[i1] = mul(sub_lazy(u, v), w);
    }
    __syncthreads();
  }
}

// Inverse transform of natural-order values to natural-order coefficients
// (scaled by 1/n), in place; one block per lane, lanes[blockIdx.x].
// n >= 16: DIT whose first pass gathers the bit-reversed input from global
// memory; smaller n: radix-2 stages in shared memory.
// LOGN: the size when fixed at compile time (2^4..2^14), else 0 and logn_rt.
template <int LOGN>
__global__ void k_intt(uint32_t* const* lanes, int logn_rt, const uint32_t* tw_n, uint32_t n_inv) {
  const int logn = LOGN ? LOGN : logn_rt;
  extern __shared__ uint32_t sm[];
  const uint32_t n = 1u << logn;
  uint32_t* d = lanes[blockIdx.x];
  if (logn < 4) {
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) sm[bitrev32(k, logn)] = d[k];
    __syncthreads();
    smem_dit(sm, logn, tw_n, true);
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) d[k] = mul(sm[k], n_inv);
    return;
  }
  auto first = [&](uint32_t t, uint32_t r, int lo) { return d[bitrev32(grp_index(t, r, lo), logn)]; };
  auto store = [&](uint32_t t, int lo, const uint32_t* v) {
#pragma unroll
    for (uint32_t r = 0; r < 16; r++) d[grp_index(t, r, lo)] = mul(v[r], n_inv);
  };
  ntt16<false>(sm, logn, tw_n, true, first, store);
}

// LDE of one lane per block: Lagrange values in natural order (or canonical
// coefficients when from_coeffs) -> for coset a < 4,
// out[a n + b] = P(w_4n^bitrev2(a) w_n^bitrev(b)), the bit-reversed
// evaluations on <w_4n> of reedsolomon.Encode (internal/reedsolomon/rs.go:52-70).
// Optionally writes the coefficients.  Shared memory: A (coefficients) and B
// (work), pad16 layout.
// 4-byte asynchronous copy global -> shared (cp.async, no register staging):
// a thread issues all of its copies before waiting for any.
__device__ __forceinline__ void cp_async4(uint32_t* smem, const uint32_t* gmem) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

struct LdeLane { const uint32_t* src; uint32_t* out; uint32_t* coef; };
// fwd = 0: only the inverse transform, coset 0 and the coefficients (L.coef,
// which must be set); k_lde_fwd then runs the other cosets.
template <int LOGN>
__global__ void k_lde(const LdeLane* lanes, int logn_rt, int from_coeffs, const uint32_t* tw_n, const uint32_t* tw_4n,
                      uint32_t n_inv, int fwd = 1) {
  const int logn = LOGN ? LOGN : logn_rt;
  extern __shared__ uint32_t sm[];
  const uint32_t n = 1u << logn;
  const LdeLane L = lanes[blockIdx.x];
  const uint32_t big = n << RATE_LOG;
  if (logn < 4) {  // tiny columns: radix-2 stages
    uint32_t* A = sm;
    uint32_t* B = sm + n;
    if (from_coeffs) {
      for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) A[k] = L.src[k];
      __syncthreads();
    } else {
      for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) A[bitrev32(k, logn)] = L.src[k];
      __syncthreads();
      smem_dit(A, logn, tw_n, true);
      for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) A[k] = mul(A[k], n_inv);
      __syncthreads();
    }
    if (L.coef)
      for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) L.coef[k] = A[k];
    for (int a = 0; a < (1 << RATE_LOG); a++) {
      const uint32_t e = bitrev32((uint32_t)a, RATE_LOG);
      for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) B[k] = mul(A[k], __ldg(tw_4n + ((e * k) & (big - 1))));
      __syncthreads();
      smem_dif(B, logn, tw_n, false);
      for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) L.out[(uint64_t)a * n + k] = B[k];
      __syncthreads();
    }
    return;
  }
  uint32_t* A = sm;
  uint32_t* B = sm + pad16(n);
  if (from_coeffs) {
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
      uint32_t v = L.src[k];
      A[pad16(k)] = v;
      if (L.coef) L.coef[k] = v;
    }
    __syncthreads();
  } else {
    // the input goes to B (free until the coset transforms) with coalesced
    // loads; the first pass gathers it in bit-reversed order from there
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) B[pad16(k)] = L.src[k];
    __syncthreads();
    auto first = [&](uint32_t t, uint32_t r, int lo) { return B[pad16(bitrev32(grp_index(t, r, lo), logn))]; };
    auto store = [&](uint32_t t, int lo, const uint32_t* v) {
#pragma unroll
      for (uint32_t r = 0; r < 16; r++) {
        uint32_t i = grp_index(t, r, lo), c = mul(v[r], n_inv);
        A[pad16(i)] = c;
        if (L.coef) L.coef[i] = c;
      }
    };
    // Coset 0 is <w_n> itself: its bit-reversed evaluations are the input
    // values in bit-reversed order, which the DIT's first pass (local bits
    // [0, 4): 16 consecutive positions) has just gathered.
    auto coset0 = [&](uint32_t t, const uint32_t* v) {
      uint4* q = reinterpret_cast<uint4*>(L.out + ((uint64_t)t << 4));
      q[0] = make_uint4(v[0], v[1], v[2], v[3]);
      q[1] = make_uint4(v[4], v[5], v[6], v[7]);
      q[2] = make_uint4(v[8], v[9], v[10], v[11]);
      q[3] = make_uint4(v[12], v[13], v[14], v[15]);
    };
    ntt16<false>(A, logn, tw_n, true, first, store, coset0);  // A is both work and result
  }
  if (!fwd) return;
  for (int a = from_coeffs ? 0 : 1; a < (1 << RATE_LOG); a++) {
    const uint32_t e = bitrev32((uint32_t)a, RATE_LOG);
    uint32_t* o = L.out + (uint64_t)a * n;
    auto first = [&](uint32_t t, uint32_t r, int lo) {
      uint32_t i = grp_index(t, r, lo);
      return mul(A[pad16(i)], __ldg(tw_4n + ((e * i) & (big - 1))));
    };
    auto store = [&](uint32_t t, int lo, const uint32_t* v) {
      // DIF's last pass has lo = 0: the group is 16 consecutive outputs
      uint4* q = reinterpret_cast<uint4*>(o + ((uint64_t)t << 4));
      q[0] = make_uint4(v[0], v[1], v[2], v[3]);
      q[1] = make_uint4(v[4], v[5], v[6], v[7]);
      q[2] = make_uint4(v[8], v[9], v[10], v[11]);
      q[3] = make_uint4(v[12], v[13], v[14], v[15]);
    };
    ntt16<true>(B, logn, tw_n, false, first, store);
  }
}

// The coset transforms of the LDE as blocks of their own: block (x, y) runs
// coset a = first + x of lane lane0 + y (the cosets of a lane side by side,
// so its coefficients come from DRAM once and from L2 after) from its
// coefficients (L.coef, or L.src when
// the lane is given as coefficients), written bit-reversed as in k_lde.  One
// shared-memory array per block (the coefficients are read from global
// memory, where the inverse transform left them, rather than kept in shared
// memory), so several blocks share an SM and overlap one another's barriers
// and shared-memory round trips.  MAXT: the block size the kernel is built
// for (registers capped so that 1024 / MAXT blocks fit: 32 warps per SM
// without spills).
// The coset shifts of the first DIF pass: its element i = r 2^(logn-4) + t
// (t < 2^(logn-4)) takes w_4n^(e i) = w_4n^(e t) w_64^(e r), since
// w_4n^(2^(logn-4)) = w_64 for every size; w_64^(e r) for e < 4, r < 16 as
// canonical words with their Shoup companions.
struct CosetSteps { uint32_t w[4][16], ws[4][16]; };
constexpr CosetSteps make_coset_steps() {
  CosetSteps c{};
  for (uint32_t e = 0; e < 4; e++)
    for (uint32_t r = 0; r < 16; r++) {
      c.w[e][r] = cx_pow(3, (uint64_t)((P - 1) / 64) * ((e * r) % 64));
      c.ws[e][r] = shoup(c.w[e][r]);
    }
  return c;
}
__constant__ CosetSteps COSET_STEPS_D = make_coset_steps();

template <int LOGN, int MAXT>
__global__ void __launch_bounds__(MAXT, 1024 / MAXT)
    k_lde_fwd(const LdeLane* lanes, uint32_t lane0, int first, const uint32_t* tw_n, const uint32_t* tw_4n) {
  static_assert(LOGN >= 4, "radix-16 passes");
  extern __shared__ uint32_t sm[];
  constexpr uint32_t n = 1u << LOGN, big = n << RATE_LOG;
  const LdeLane L = lanes[lane0 + blockIdx.y];
  const uint32_t a = first + blockIdx.x;
  const uint32_t e = bitrev32(a, RATE_LOG);
  const uint32_t* coef = L.coef ? L.coef : L.src;
  uint32_t* o = L.out + (uint64_t)a * n;
  // the coefficients go to shared memory first (cp.async, coalesced, all in
  // flight at once); the first pass reads and overwrites its own positions
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) cp_async4(&sm[pad16(k)], coef + k);
  cp_async_wait_all();
  __syncthreads();
  // one table load per group for w_4n^(e t); the 15 other shifts of the group
  // are Shoup products by constants (r is a compile-time index after unrolling)
  uint32_t shift_t = 0;
  auto first_pass = [&](uint32_t t, uint32_t r, int lo) {
    const uint32_t i = grp_index(t, r, lo);
    if (r == 0) shift_t = __ldg(tw_4n + ((e * t) & (big - 1)));
    const uint32_t x = mul(sm[pad16(i)], shift_t);
    return r ? mulc(x, COSET_STEPS_D.w[e][r], COSET_STEPS_D.ws[e][r]) : x;
  };
  auto store = [&](uint32_t t, int lo, const uint32_t* v) {
    uint4* q = reinterpret_cast<uint4*>(o + ((uint64_t)t << 4));
    q[0] = make_uint4(v[0], v[1], v[2], v[3]);
    q[1] = make_uint4(v[4], v[5], v[6], v[7]);
    q[2] = make_uint4(v[8], v[9], v[10], v[11]);
    q[3] = make_uint4(v[12], v[13], v[14], v[15]);
  };
  ntt16<true>(sm, LOGN, tw_n, false, first_pass, store);
}

// The inverse transform of the split LDE, one lane per block with a single
// shared-memory array: the first pass gathers its bit-reversed inputs from
// global memory (the lane's few tens of KB stay in L1 while the block reads
// them), writes coset 0 (the input in bit-reversed order) from those
// registers, and the last pass writes the coefficients to global memory,
// where k_lde_fwd reads them.
template <int LOGN, int MAXT>
__global__ void __launch_bounds__(MAXT, 1024 / MAXT)
    k_lde_inv(const LdeLane* lanes, const uint32_t* tw_n, uint32_t n_inv) {
  static_assert(LOGN >= 4, "radix-16 passes");
  extern __shared__ uint32_t sm[];
  const LdeLane L = lanes[blockIdx.x];
  auto first = [&](uint32_t t, uint32_t r, int lo) { return __ldg(L.src + bitrev32(grp_index(t, r, lo), LOGN)); };
  auto coset0 = [&](uint32_t t, const uint32_t* v) {
    uint4* q = reinterpret_cast<uint4*>(L.out + ((uint64_t)t << 4));
    q[0] = make_uint4(v[0], v[1], v[2], v[3]);
    q[1] = make_uint4(v[4], v[5], v[6], v[7]);
    q[2] = make_uint4(v[8], v[9], v[10], v[11]);
    q[3] = make_uint4(v[12], v[13], v[14], v[15]);
  };
  auto store = [&](uint32_t t, int lo, const uint32_t* v) {
#pragma unroll
    for (uint32_t r = 0; r < 16; r++) L.coef[grp_index(t, r, lo)] = mul(v[r], n_inv);
  };
  ntt16<false>(sm, LOGN, tw_n, true, first, store, coset0);
}

// Evaluations of a coefficient lane on the cosets s_c <w_n>, s_c = g w_4n^c,
// c = blockIdx.y < 4, in natural order: out[c n + j] = P(s_c w_n^j).
// n >= 16: the scaled coefficients coef[k] s_c^k (shift: the table of s_c^k,
// coset_shifts) go to the second half of shared memory with coalesced loads;
// a DIT whose first pass gathers them in bit-reversed order from there works
// in the first half.
struct CosetLane { const uint32_t* src; uint32_t* out; };
template <int LOGN>
__global__ void k_coset_eval(const CosetLane* lanes, int logn_rt, const uint32_t* tw_n, const uint32_t* shift) {
  const int logn = LOGN ? LOGN : logn_rt;
  extern __shared__ uint32_t sm[];
  const uint32_t n = 1u << logn, c = blockIdx.y;
  const CosetLane L = lanes[blockIdx.x];
  const uint32_t* sh = shift + (uint64_t)c * n;
  uint32_t* o = L.out + (uint64_t)c * n;
  if (logn < 4) {
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) sm[k] = mul(L.src[k], sh[k]);
    __syncthreads();
    smem_dif(sm, logn, tw_n, false);
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) o[j] = sm[bitrev32(j, logn)];
    return;
  }
  // the coefficients (to S2) and the shift powers (to the work half, free
  // until the first pass) arrive by cp.async, all copies in flight at once;
  // then each thread scales its own words
  uint32_t* S2 = sm + pad16(n) + 1;
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
    cp_async4(&S2[pad16(k)], L.src + k);
    cp_async4(&sm[pad16(k)], sh + k);
  }
  cp_async_wait_all();
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) S2[pad16(k)] = mul(S2[pad16(k)], sm[pad16(k)]);
  __syncthreads();
  auto first = [&](uint32_t t, uint32_t r, int lo) { return S2[pad16(bitrev32(grp_index(t, r, lo), logn))]; };
  auto store = [&](uint32_t t, int lo, const uint32_t* v) {
#pragma unroll
    for (uint32_t r = 0; r < 16; r++) o[grp_index(t, r, lo)] = v[r];
  };
  ntt16<false>(sm, logn, tw_n, false, first, store);
}

// ---------------------------------------------------------------- leaves
// leaf k = Sponge(LEAF, 2nB, 2nE, lo.base, hi.base, lo.ext, hi.ext) over
// rows 2k, 2k+1 (internal/fri/hash.go:39-57).  Base lanes at base + c*stride,
// ext column e lane l at ext + (6e + l)*stride.
struct LeafGroup {
  const uint32_t* base;
  const uint32_t* ext;
  uint64_t stride;      // words between lanes
  uint32_t nb, ne;
  uint32_t n_leaves;    // rows / 2
  uint32_t* out;        // n_leaves digests of 8 words
};

__device__ __forceinline__ uint32_t leaf_elem(const LeafGroup& g, uint32_t idx, uint32_t k, uint32_t hdr0,
                                              uint32_t hdr1, uint32_t hdr2) {
  if (idx == 0) return hdr0;
  if (idx == 1) return hdr1;
  if (idx == 2) return hdr2;
  idx -= 3;
  if (idx < 2 * g.nb) {
    uint32_t h = idx >= g.nb;
    uint32_t c = idx - h * g.nb;
    return g.base[c * g.stride + 2 * k + h];
  }
  idx -= 2 * g.nb;
  uint32_t h = idx >= 6 * g.ne;
  uint32_t e = idx - h * 6 * g.ne;
  return g.ext[e * g.stride + 2 * k + h];
}

// One thread per leaf: the fewest instructions per permutation, for launches
// with enough leaves to fill the GPU.
__global__ void k_hash_leaves1(const LeafGroup* groups) {
  const LeafGroup g = groups[blockIdx.y];
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= g.n_leaves) return;
  const uint32_t total = 3 + 2 * g.nb + 12 * g.ne;
  const uint32_t h0 = to_mont(LEAF_TAG), h1 = to_mont(2 * g.nb), h2 = to_mont(2 * g.ne);
  uint32_t s[24];
#pragma unroll
  for (int i = 0; i < 24; i++) s[i] = 0;
  for (uint32_t b = 0; b < total; b += 16) {
#pragma unroll
    for (uint32_t i = 0; i < 16; i++)
      if (b + i < total) s[i] = leaf_elem(g, b + i, k, h0, h1, h2);
    p2_permute(s);
  }
  uint32_t* o = g.out + (uint64_t)k * 8;
#pragma unroll
  for (int i = 0; i < 8; i++) o[i] = s[i];
}

// Cooperative form: six lanes per leaf (p2_coop.cuh), five leaves per warp.
constexpr uint32_t P2_GROUPS_PER_WARP = 5;

__global__ void k_hash_leaves(const LeafGroup* groups) {
  __shared__ uint32_t keys[144];
  p2_load_full_keys(keys);
  P2Lane L;
  L.init();
  const LeafGroup g = groups[blockIdx.y];
  const uint32_t warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  const uint32_t k = (blockIdx.x * warps + warp) * P2_GROUPS_PER_WARP + (uint32_t)L.base / 6;
  const bool active = L.lane < 30 && k < g.n_leaves;
  const uint32_t total = 3 + 2 * g.nb + 12 * g.ne;
  const uint32_t h0 = to_mont(LEAF_TAG), h1 = to_mont(2 * g.nb), h2 = to_mont(2 * g.ne);
  uint32_t x[4] = {0, 0, 0, 0};
  for (uint32_t b = 0; b < total; b += 16) {
    if (active && L.idx < 4) {
#pragma unroll
      for (uint32_t i = 0; i < 4; i++) {
        uint32_t e = b + 4 * L.idx + i;
        if (e < total) x[i] = leaf_elem(g, e, k, h0, h1, h2);
      }
    }
    p2c_permute(x, L, keys);
  }
  if (active && L.idx < 2) {
    uint32_t* o = g.out + (uint64_t)k * 8 + 4 * L.idx;
#pragma unroll
    for (int i = 0; i < 4; i++) o[i] = x[i];
  }
}

// ---------------------------------------------------------------- Merkle
// nodes: 1-indexed, 8 words per node.  Level step: node i = H(2i, 2i+1) for
// i in [start, 2 start); injection fold: node start+j = H(node, inj[j]),
// several injections of the same width chained in schedule order
// (internal/merkle/tree.go:210-327).  Six lanes per node.

// Loads digest words into the left (idx 2, 3) or right (idx 4, 5) slot.
__device__ __forceinline__ void p2c_load_slot(uint32_t x[4], const P2Lane& L, int slot, const uint32_t* digest,
                                              bool active) {
  if (active && (L.idx >> 1) == slot) {
    const uint32_t* d = digest + 4 * (L.idx & 1);
#pragma unroll
    for (int i = 0; i < 4; i++) x[i] = d[i];
  }
}
__device__ __forceinline__ void p2c_store_digest(const uint32_t x[4], const P2Lane& L, uint32_t* digest, bool active) {
  if (active && L.idx < 2) {
    uint32_t* d = digest + 4 * L.idx;
#pragma unroll
    for (int i = 0; i < 4; i++) d[i] = x[i];
  }
}

__device__ __forceinline__ void merkle_node(uint32_t* nodes, uint64_t id, const P2Lane& L, const uint32_t* keys,
                                            bool active) {
  uint32_t x[4] = {0, 0, 0, 0};
  p2c_load_slot(x, L, 1, nodes + 2 * id * 8, active);
  p2c_load_slot(x, L, 2, nodes + (2 * id + 1) * 8, active);
  p2c_compress(x, L, keys);
  p2c_store_digest(x, L, nodes + id * 8, active);
}

// node = H(... H(H(node, inj_0[j]), inj_1[j]) ..., inj_{n-1}[j])
__device__ __forceinline__ void merkle_chain(uint32_t* nodes, uint64_t id, uint32_t j, const uint32_t* const* inj,
                                             uint32_t n_inj, const P2Lane& L, const uint32_t* keys, bool active) {
  if (n_inj == 0) return;
  uint32_t x[4] = {0, 0, 0, 0};
  p2c_load_slot(x, L, 1, nodes + id * 8, active);
  for (uint32_t t = 0; t < n_inj; t++) {
    p2c_load_slot(x, L, 2, inj[t] + (uint64_t)j * 8, active);
    p2c_compress(x, L, keys);
    if (t + 1 < n_inj) p2c_digest_to_left(x, L);
  }
  p2c_store_digest(x, L, nodes + id * 8, active);
}

__global__ void k_merkle_level(uint32_t* nodes, uint32_t start) {
  __shared__ uint32_t keys[144];
  p2_load_full_keys(keys);
  P2Lane L;
  L.init();
  const uint32_t warps = blockDim.x >> 5;
  const uint32_t i = (blockIdx.x * warps + (threadIdx.x >> 5)) * P2_GROUPS_PER_WARP + (uint32_t)L.base / 6;
  merkle_node(nodes, (uint64_t)start + i, L, keys, L.lane < 30 && i < start);
}

__global__ void k_merkle_inject(uint32_t* nodes, uint32_t start, const uint32_t* const* inj, uint32_t n_inj) {
  __shared__ uint32_t keys[144];
  p2_load_full_keys(keys);
  P2Lane L;
  L.init();
  const uint32_t warps = blockDim.x >> 5;
  const uint32_t j = (blockIdx.x * warps + (threadIdx.x >> 5)) * P2_GROUPS_PER_WARP + (uint32_t)L.base / 6;
  merkle_chain(nodes, (uint64_t)start + j, j, inj, n_inj, L, keys, L.lane < 30 && j < start);
}

// One thread per node (levels and injection chains wide enough to fill the
// GPU): the fewest instructions per permutation.  Digests are 32-byte
// aligned, so they move as two 16-byte words.
__device__ __forceinline__ void ld_digest(const uint32_t* p, uint32_t d[8]) {
  const uint4 a = reinterpret_cast<const uint4*>(p)[0], b = reinterpret_cast<const uint4*>(p)[1];
  d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w; d[4] = b.x; d[5] = b.y; d[6] = b.z; d[7] = b.w;
}
__device__ __forceinline__ void st_digest(uint32_t* p, const uint32_t d[8]) {
  reinterpret_cast<uint4*>(p)[0] = make_uint4(d[0], d[1], d[2], d[3]);
  reinterpret_cast<uint4*>(p)[1] = make_uint4(d[4], d[5], d[6], d[7]);
}
__global__ void k_merkle_level1(uint32_t* nodes, uint32_t start) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= start) return;
  const uint64_t id = (uint64_t)start + i;
  uint32_t l[8], r[8];
  ld_digest(nodes + 2 * id * 8, l);
  ld_digest(nodes + (2 * id + 1) * 8, r);
  p2_compress(to_mont(NODE_TAG), l, r, l);
  st_digest(nodes + id * 8, l);
}
__global__ void k_merkle_inject1(uint32_t* nodes, uint32_t start, const uint32_t* const* inj, uint32_t n_inj) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= start) return;
  uint32_t* nd = nodes + ((uint64_t)start + j) * 8;
  uint32_t l[8], r[8];
  ld_digest(nd, l);
  for (uint32_t t = 0; t < n_inj; t++) {
    ld_digest(inj[t] + (uint64_t)j * 8, r);
    p2_compress(to_mont(NODE_TAG), l, r, l);
  }
  st_digest(nd, l);
}

// Upper tree levels, one subtree per block: block b of B (gridDim.x) owns the
// nodes [b top/B, (b+1) top/B) of width `top` and, for each width w from
// top/2 down to B, runs the 2-to-1 step over its share of the level, then the
// injections of width w in schedule order, with a block barrier between
// levels.  One block (B = 1) builds a whole tree top; B > 1 replaces the
// launches of the levels top/2 .. B, which are latency bound, by one.  When
// fold_first, the injections of width `top` fold first (a tree whose leaf
// level fits in one block).
// With fs.out set (one block only), the block then hashes the challenge that
// binds the root: fs.out = sponge(fs.pre[0..n_pre) || fs.prev[0..8) || root),
// as k_fs_challenge, which it replaces for the FRI layer trees.
struct InjRef { const uint32_t* leaves; uint32_t width; };
struct FsTail { const uint32_t* pre; uint32_t n_pre; const uint32_t* prev; uint32_t* out; };
__global__ void k_merkle_tail(uint32_t* nodes, uint32_t top, int fold_first, const InjRef* inj, uint32_t n_inj,
                              FsTail fs) {
  __shared__ uint32_t keys[144];
  __shared__ const uint32_t* chain[64];
  __shared__ uint32_t msg[64];
  p2_load_full_keys(keys);
  P2Lane L;
  L.init();
  const uint32_t warp = threadIdx.x >> 5, warps = blockDim.x >> 5, per = warps * P2_GROUPS_PER_WARP;
  const uint32_t nb = gridDim.x, b = blockIdx.x, slot = warp * P2_GROUPS_PER_WARP + (uint32_t)L.base / 6;
  auto fold = [&](uint32_t w) {
    uint32_t cnt = 0;
    for (uint32_t t = 0; t < n_inj && cnt < 64; t++)
      if (inj[t].width == w) {
        if (threadIdx.x == 0) chain[cnt] = inj[t].leaves;
        cnt++;
      }
    __syncthreads();
    const uint32_t share = w / nb;
    if (cnt)
      for (uint32_t j0 = 0; j0 < share; j0 += per) {
        const uint32_t jl = j0 + slot, j = b * share + jl;
        merkle_chain(nodes, (uint64_t)w + j, j, chain, cnt, L, keys, L.lane < 30 && jl < share);
      }
    __syncthreads();
  };
  if (fold_first) fold(top);
  for (uint32_t w = top >> 1; w >= nb; w >>= 1) {
    const uint32_t share = w / nb;
    for (uint32_t i0 = 0; i0 < share; i0 += per) {
      const uint32_t il = i0 + slot;
      merkle_node(nodes, (uint64_t)w + b * share + il, L, keys, L.lane < 30 && il < share);
    }
    __syncthreads();
    fold(w);
  }
  if (fs.out && warp == 0) {  // the root is nodes[1], written before the last barrier
    const uint32_t total = fs.n_pre + 16;
    for (uint32_t i = L.lane; i < total; i += 32)
      msg[i] = i < fs.n_pre ? fs.pre[i] : (i < fs.n_pre + 8 ? fs.prev[i - fs.n_pre] : nodes[8 + i - fs.n_pre - 8]);
    __syncwarp();
    uint32_t x[4] = {0, 0, 0, 0};
    for (uint32_t b0 = 0; b0 < total; b0 += 16) {
      const uint32_t len = min(16u, total - b0);
      if (L.idx < 4)
#pragma unroll
        for (int k = 0; k < 4; k++)
          if (4 * (uint32_t)L.idx + k < len) x[k] = msg[b0 + 4 * L.idx + k];
      p2c_permute(x, L, keys);
    }
    if (L.lane < 2)
#pragma unroll
      for (int k = 0; k < 4; k++) fs.out[4 * L.lane + k] = x[k];
  }
}

// Permutation test hook: one state of 24 words per group of six lanes.
__global__ void k_p2_permute(uint32_t* states, uint64_t n) {
  __shared__ uint32_t keys[144];
  p2_load_full_keys(keys);
  P2Lane L;
  L.init();
  const uint64_t warps = blockDim.x >> 5;
  const uint64_t i = (blockIdx.x * warps + (threadIdx.x >> 5)) * P2_GROUPS_PER_WARP + (uint64_t)L.base / 6;
  const bool active = L.lane < 30 && i < n;
  uint32_t x[4] = {0, 0, 0, 0};
  if (active)
    for (int q = 0; q < 4; q++) x[q] = states[i * 24 + 4 * L.idx + q];
  p2c_permute(x, L, keys);
  if (active)
    for (int q = 0; q < 4; q++) states[i * 24 + 4 * L.idx + q] = x[q];
}

// ---------------------------------------------------------------- expressions
// Register bytecode for the constraint DAG (compiled on the host from the
// program's folded relation): typed ops over a per-thread register file of
// E6 slots held in shared memory.
enum : uint8_t {
  X_LOAD_B = 0,  // r[d] = col lane imm at row (j + shift) mod n (base)
  X_LOAD_E,      // r[d] = 6 lanes starting at lane imm (ext)
  X_COIN,        // r[d] = coins[imm]
  X_CONST,       // r[d] = imm (base, Montgomery)
  X_ADD_BB, X_ADD_EB, X_ADD_EE,
  X_SUB_BB, X_SUB_BE, X_SUB_EB, X_SUB_EE,
  X_MUL_BB, X_MUL_EB, X_MUL_EE,
};
struct XInst { uint8_t op, d, a, b; uint32_t imm; int32_t shift; };
constexpr int X_MAX_REGS = 24;
constexpr int X_MAX_INST = 16384;  // instructions are read from global memory; no fixed array

struct XProgram {
  const XInst* code;
  uint32_t n_inst;
  uint32_t n_regs;
  uint32_t result;      // register holding the value
  uint32_t result_ext;  // 1 when the result is an E6
};

// Evaluates one row.  lane(l, row) returns column lane l at `row`.
template <class LaneFn>
__device__ __forceinline__ E6 x_eval(const XProgram& p, const E6* coins, uint32_t* regs, uint32_t stride, uint32_t j,
                                     uint32_t n, LaneFn lane) {
  // regs: register r word w at regs[(r * 6 + w) * stride]
  auto R = [&](uint32_t r, int w) -> uint32_t& { return regs[(r * 6 + w) * stride]; };
  for (uint32_t pc = 0; pc < p.n_inst; pc++) {
    XInst in = p.code[pc];
    switch (in.op) {
      case X_LOAD_B: {
        uint32_t row = (uint32_t)(((int64_t)j + in.shift) & (int64_t)(n - 1));
        R(in.d, 0) = lane(in.imm, row);
        break;
      }
      case X_LOAD_E: {
        uint32_t row = (uint32_t)(((int64_t)j + in.shift) & (int64_t)(n - 1));
        for (int w = 0; w < 6; w++) R(in.d, w) = lane(in.imm + w, row);
        break;
      }
      case X_COIN:
        for (int w = 0; w < 6; w++) R(in.d, w) = coins[in.imm].c[w];
        break;
      case X_CONST: R(in.d, 0) = in.imm; break;
      case X_ADD_BB: R(in.d, 0) = add(R(in.a, 0), R(in.b, 0)); break;
      case X_ADD_EB: {  // a ext, b base
        uint32_t b0 = R(in.b, 0);
        for (int w = 1; w < 6; w++) R(in.d, w) = R(in.a, w);
        R(in.d, 0) = add(R(in.a, 0), b0);
        break;
      }
      case X_ADD_EE: for (int w = 0; w < 6; w++) R(in.d, w) = add(R(in.a, w), R(in.b, w)); break;
      case X_SUB_BB: R(in.d, 0) = sub(R(in.a, 0), R(in.b, 0)); break;
      case X_SUB_BE: {  // a base, b ext
        uint32_t a0 = R(in.a, 0);
        for (int w = 1; w < 6; w++) R(in.d, w) = neg(R(in.b, w));
        R(in.d, 0) = sub(a0, R(in.b, 0));
        break;
      }
      case X_SUB_EB: {
        uint32_t b0 = R(in.b, 0);
        for (int w = 1; w < 6; w++) R(in.d, w) = R(in.a, w);
        R(in.d, 0) = sub(R(in.a, 0), b0);
        break;
      }
      case X_SUB_EE: for (int w = 0; w < 6; w++) R(in.d, w) = sub(R(in.a, w), R(in.b, w)); break;
      case X_MUL_BB: R(in.d, 0) = mul(R(in.a, 0), R(in.b, 0)); break;
      case X_MUL_EB: {
        uint32_t b0 = R(in.b, 0);
        for (int w = 0; w < 6; w++) R(in.d, w) = mul(R(in.a, w), b0);
        break;
      }
      case X_MUL_EE: {
        E6 x, y;
        for (int w = 0; w < 6; w++) { x.c[w] = R(in.a, w); y.c[w] = R(in.b, w); }
        E6 z = e6_mul(x, y);
        for (int w = 0; w < 6; w++) R(in.d, w) = z.c[w];
        break;
      }
    }
  }
  E6 r;
  if (p.result_ext) { for (int w = 0; w < 6; w++) r.c[w] = R(p.result, w); }
  else r = e6_base(R(p.result, 0));
  return r;
}

// Quotient numerator of one module on coset c = blockIdx.y, row j:
// V(...) / (s_c^n - 1), written as qv[w * 4n + c n + j].  cv: coset values,
// lane l coset c at cv[l * 4n + c n + j].  One job per module (blockIdx.z).
struct QJob { XProgram p; const uint32_t* cv; uint32_t* qv; int logn; uint32_t zinv[4]; };
__global__ void k_quotient_eval(const QJob* jobs, const E6* coins) {
  extern __shared__ uint32_t regs[];
  const QJob& J = jobs[blockIdx.z];
  const uint32_t n = 1u << J.logn;
  const uint32_t c = blockIdx.y;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint64_t big = (uint64_t)n << RATE_LOG;
  const uint32_t* cv = J.cv;
  auto lane = [&](uint32_t l, uint32_t row) -> uint32_t { return cv[l * big + (uint64_t)c * n + row]; };
  E6 v = x_eval(J.p, coins, regs + threadIdx.x, blockDim.x, j, n, lane);
  v = e6_mul_base(v, J.zinv[c]);
  uint32_t lw = J.p.result_ext ? 6 : 1;
  for (uint32_t w = 0; w < lw; w++) J.qv[w * big + (uint64_t)c * n + j] = v.c[w];
}

// Quotient chunk coefficients from the inverse-transformed coset values.
// r[w][c n + k] holds [Y^k] R_c(Y), R_c(Y) = sum_d s_c^(dn) q_d(s_c Y).
// With t_c = r_c[k] s_c^-k, u_d = g^(dn) q_(d,k) = 1/4 sum_c t_c w_4^(-cd).
// out: chunk d, lane w at out[(d * lanes + w) * n + k].  One job per module.
struct QcJob { const uint32_t* r; uint32_t* out; int logn; uint32_t lanes; const uint32_t* ginv_pow; const uint32_t* tw_4n; uint32_t gn_inv; };
__global__ void k_quotient_chunks(const QcJob* jobs, uint32_t quarter) {
  const QcJob& J = jobs[blockIdx.z];
  const uint32_t n = 1u << J.logn;
  const uint64_t big = (uint64_t)n << RATE_LOG;
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t w = blockIdx.y;
  if (k >= n || w >= J.lanes) return;
  uint32_t t[4];
  const uint32_t gk = J.ginv_pow[k];
  for (int c = 0; c < 4; c++) {
    uint32_t e = (uint32_t)((big - ((uint64_t)c * k) % big) % big);  // s_c^-k = g^-k w_4n^-(c k)
    t[c] = mul(mul(J.r[w * big + (uint64_t)c * n + k], gk), __ldg(J.tw_4n + e));
  }
  const uint32_t w4i = __ldg(J.tw_4n + 3 * n), w4i2 = mul(w4i, w4i), w4i3 = mul(w4i2, w4i);
  uint32_t u[4];
  u[0] = add(add(t[0], t[1]), add(t[2], t[3]));
  u[1] = add(add(t[0], mul(t[1], w4i)), add(mul(t[2], w4i2), mul(t[3], w4i3)));
  u[2] = add(add(t[0], mul(t[1], w4i2)), add(t[2], mul(t[3], w4i2)));
  u[3] = add(add(t[0], mul(t[1], w4i3)), add(mul(t[2], w4i2), mul(t[3], w4i)));
  uint32_t scale = quarter;
  for (int d = 0; d < 4; d++) {
    J.out[((uint64_t)d * J.lanes + w) * n + k] = mul(u[d], scale);
    scale = mul(scale, J.gn_inv);
  }
}

// ---------------------------------------------------------------- grand product
// ratio[j] = num(j) / den(j) on Lagrange rows (internal/poly/iop_utils.go:170-192).
// One job per step (blockIdx.y); lanes[l] is lane l of the step's inputs.
struct GpJob { XProgram pn, pd; const uint32_t* const* lanes; uint32_t* ratio; int logn; };
__global__ void k_gp_ratio(const GpJob* jobs, const E6* coins) {
  extern __shared__ uint32_t regs[];
  const GpJob& J = jobs[blockIdx.y];
  const uint32_t n = 1u << J.logn;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t* const* lanes = J.lanes;
  auto lane = [&](uint32_t l, uint32_t row) -> uint32_t { return lanes[l][row]; };
  E6 a = x_eval(J.pn, coins, regs + threadIdx.x, blockDim.x, j, n, lane);
  E6 b = x_eval(J.pd, coins, regs + threadIdx.x, blockDim.x, j, n, lane);
  E6 q = e6_mul(a, e6_inv(b));
  for (int w = 0; w < 6; w++) J.ratio[(uint64_t)w * n + j] = q.c[w];
}

constexpr int SCAN_BLOCK = 256, SCAN_PER_THREAD = 8, SCAN_TILE = SCAN_BLOCK * SCAN_PER_THREAD;

__device__ __forceinline__ E6 ld6(const uint32_t* p, uint64_t stride, uint64_t i) {
  E6 r;
  for (int w = 0; w < 6; w++) r.c[w] = p[w * stride + i];
  return r;
}
__device__ __forceinline__ void st6(uint32_t* p, uint64_t stride, uint64_t i, const E6& v) {
  for (int w = 0; w < 6; w++) p[w * stride + i] = v.c[w];
}

// Product scans over E6 vectors stored as 6 lanes of n words: per-tile
// inclusive scan in place, tile totals, their exclusive prefix, and the
// shifted result out[0] = 1, out[i] = prod_{k<i} x[k].  One job per vector.
struct ScanJob {
  uint32_t* x;
  uint64_t n;
  uint32_t* totals;
  uint32_t* pre;
  uint32_t* out;
  uint32_t nt;
  uint32_t inclusive = 0;  // running ratio: out[i] = prod_{k<=i} x[k] ...
  uint32_t* end = nullptr; // ... and its last value written here (6 words)
};

// The scans run over products (grand products) or sums (logup running sums).
template <bool SUM> __device__ __forceinline__ E6 scan_id() { return SUM ? e6_zero() : e6_one(); }
template <bool SUM> __device__ __forceinline__ E6 scan_op(const E6& a, const E6& b) {
  return SUM ? e6_add(a, b) : e6_mul(a, b);
}

template <bool SUM = false>
__global__ void k_scan_tiles(const ScanJob* jobs) {
  __shared__ E6 part[SCAN_BLOCK];
  const ScanJob& J = jobs[blockIdx.y];
  if (blockIdx.x >= J.nt) return;
  const uint64_t n = J.n;
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_PER_THREAD;
  E6 acc = scan_id<SUM>();
  E6 v[SCAN_PER_THREAD];
  for (int i = 0; i < SCAN_PER_THREAD; i++) {
    uint64_t idx = base + i;
    v[i] = idx < n ? ld6(J.x, n, idx) : scan_id<SUM>();
    acc = scan_op<SUM>(acc, v[i]);
    v[i] = acc;
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int off = 1; off < SCAN_BLOCK; off <<= 1) {
    E6 t = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : scan_id<SUM>();
    __syncthreads();
    if (threadIdx.x >= (unsigned)off) part[threadIdx.x] = scan_op<SUM>(part[threadIdx.x], t);
    __syncthreads();
  }
  E6 pre = threadIdx.x ? part[threadIdx.x - 1] : scan_id<SUM>();
  for (int i = 0; i < SCAN_PER_THREAD; i++) {
    uint64_t idx = base + i;
    if (idx < n) st6(J.x, n, idx, scan_op<SUM>(pre, v[i]));
  }
  if (threadIdx.x == SCAN_BLOCK - 1)
    for (int w = 0; w < 6; w++) J.totals[w * J.nt + blockIdx.x] = part[SCAN_BLOCK - 1].c[w];
}

// Exclusive prefix (products or sums) of the tile totals (one thread per
// job; nt is n / 2048).
template <bool SUM = false>
__global__ void k_tile_prefix(const ScanJob* jobs, uint32_t n_jobs) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_jobs) return;
  const ScanJob& J = jobs[i];
  E6 acc = scan_id<SUM>();
  for (uint32_t t = 0; t < J.nt; t++) {
    for (int w = 0; w < 6; w++) J.pre[t * 6 + w] = acc.c[w];
    E6 v;
    for (int w = 0; w < 6; w++) v.c[w] = J.totals[w * J.nt + t];
    acc = scan_op<SUM>(acc, v);
  }
}

__global__ void k_gp_finish(const ScanJob* jobs) {
  const ScanJob& J = jobs[blockIdx.y];
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= J.n) return;
  E6 v;
  if (!J.inclusive && i == 0) v = e6_one();
  else {
    uint64_t k = J.inclusive ? i : i - 1, tile = k / SCAN_TILE;
    E6 pre;
    for (int w = 0; w < 6; w++) pre.c[w] = J.pre[tile * 6 + w];
    v = e6_mul(pre, ld6(J.x, J.n, k));
  }
  st6(J.out, J.n, i, v);
  if (J.end && i == J.n - 1)
    for (int w = 0; w < 6; w++) J.end[w] = v.c[w];
}

// ---------------------------------------------------------------- lookups
// Cyclic logup fractions (internal/poly/iop_utils.go:110-131): per row,
// frac = sum_k M_k / E_k over the step's terms.  One job per step.
constexpr int LOGUP_MAX_TERMS = 4;
struct LogupJob {
  XProgram e[LOGUP_MAX_TERMS], m[LOGUP_MAX_TERMS];
  uint32_t n_terms;
  const uint32_t* const* lanes;
  uint32_t* frac;
  int logn;
};
__global__ void k_logup_frac(const LogupJob* jobs, const E6* coins) {
  extern __shared__ uint32_t regs[];
  const LogupJob& J = jobs[blockIdx.y];
  const uint32_t n = 1u << J.logn;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t* const* lanes = J.lanes;
  auto lane = [&](uint32_t l, uint32_t row) -> uint32_t { return lanes[l][row]; };
  E6 v = e6_zero();
  for (uint32_t k = 0; k < J.n_terms; k++) {
    E6 e = x_eval(J.e[k], coins, regs + threadIdx.x, blockDim.x, j, n, lane);
    E6 m = x_eval(J.m[k], coins, regs + threadIdx.x, blockDim.x, j, n, lane);
    v = e6_add(v, e6_mul(m, e6_inv(e)));
  }
  for (int w = 0; w < 6; w++) J.frac[(uint64_t)w * n + j] = v.c[w];
}

// L_i = S_i - (i + 1) T / n with S the inclusive running sums (tile scans in
// x plus the tile prefixes) and T = S_{n-1}; thread 0 writes T to `total`
// (board/logup.go:150-170).
struct LogupFinish { uint32_t* total; uint32_t n_inv; };
__global__ void k_logup_finish(const ScanJob* jobs, const LogupFinish* fin) {
  const ScanJob& J = jobs[blockIdx.y];
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= J.n) return;
  auto prefix = [&](uint64_t k) {
    E6 pre;
    for (int w = 0; w < 6; w++) pre.c[w] = J.pre[(k / SCAN_TILE) * 6 + w];
    return e6_add(pre, ld6(J.x, J.n, k));
  };
  const E6 T = prefix(J.n - 1);
  const E6 avg = e6_mul_base(T, fin[blockIdx.y].n_inv);
  const E6 L = e6_sub(prefix(i), e6_mul_base(avg, to_mont((uint32_t)(i + 1))));
  st6(J.out, J.n, i, L);
  if (i == 0)
    for (int w = 0; w < 6; w++) fin[blockIdx.y].total[w] = T.c[w];
}

// Lookup multiplicities of width-1 tables (internal/poly/lookup_multiplicity.go:37-100)
// with an open-addressing table per step: target values are inserted with
// the smallest combined row index (T_0 rows, then T_1 rows, ...) holding them,
// sources add one to the count of their value's first row, and the counts
// become the multiplicity columns.  A source value absent from every target
// sets `missing`.  All probe loops stop after `cap` slots.
constexpr uint32_t MULT_EMPTY = 0xffffffffu;
struct MultTab { uint32_t* keys; uint32_t* first; uint32_t* count; uint32_t cap; };
struct MultVec { const uint32_t* vals; uint32_t n, comb_off, tab; uint32_t* out; };
__device__ __forceinline__ uint32_t mult_hash(uint32_t v, uint32_t mask) {
  v ^= v >> 16;
  v *= 0x7feb352du;
  v ^= v >> 15;
  v *= 0x846ca68bu;
  v ^= v >> 16;
  return v & mask;
}
__global__ void k_mult_insert(const MultVec* tv, const MultTab* tabs) {
  const MultVec V = tv[blockIdx.y];
  const MultTab T = tabs[V.tab];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.n) return;
  const uint32_t key = V.vals[i], mask = T.cap - 1;
  uint32_t h = mult_hash(key, mask);
  for (uint32_t probe = 0; probe < T.cap; probe++, h = (h + 1) & mask) {
    const uint32_t prev = atomicCAS(T.keys + h, MULT_EMPTY, key);
    if (prev == MULT_EMPTY || prev == key) {
      atomicMin(T.first + h, V.comb_off + i);
      return;
    }
  }
}
__global__ void k_mult_count(const MultVec* sv, const MultTab* tabs, uint32_t* missing) {
  const MultVec V = sv[blockIdx.y];
  const MultTab T = tabs[V.tab];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.n) return;
  const uint32_t key = V.vals[i], mask = T.cap - 1;
  uint32_t h = mult_hash(key, mask);
  for (uint32_t probe = 0; probe < T.cap; probe++, h = (h + 1) & mask) {
    const uint32_t k = T.keys[h];
    if (k == key) {
      atomicAdd(T.count + T.first[h], 1u);
      return;
    }
    if (k == MULT_EMPTY) break;
  }
  atomicOr(missing, 1u);
}
__global__ void k_mult_write(const MultVec* tv, const MultTab* tabs) {
  const MultVec V = tv[blockIdx.y];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.n) return;
  V.out[i] = to_mont(tabs[V.tab].count[V.comb_off + i]);
}
// Tuple lookups with selectors (internal/poly/lookup_multiplicity.go:37-100).
// A step's hash table keys tuples by a representative target row whose
// tuple sits in `keys` (w words per combined target row); per slot, the
// first selected target row holding the tuple and the selected source weight
// (sum of canonical selector values, 64-bit).  Probes are bounded by the
// table size, which is at least twice the target rows.
constexpr uint32_t TUPLE_MAX_W = 8;
struct TupleVec { const uint32_t* comp[TUPLE_MAX_W]; const uint32_t* sel; uint32_t n, comb_off, tab; uint32_t* out; };
struct TupleTab { uint32_t* rep; uint32_t* first; unsigned long long* weight; uint32_t* keys; uint32_t cap, w; };
__device__ __forceinline__ uint32_t tuple_hash(const TupleVec& V, uint32_t i, uint32_t w, uint32_t mask) {
  uint32_t h = 0x9e3779b9u;
  for (uint32_t k = 0; k < w; k++) h = mult_hash(h ^ V.comp[k][i], 0xffffffffu) + k;
  return mult_hash(h, mask);
}
__device__ __forceinline__ bool tuple_eq(const TupleVec& V, uint32_t i, const uint32_t* key, uint32_t w) {
  for (uint32_t k = 0; k < w; k++)
    if (V.comp[k][i] != key[k]) return false;
  return true;
}
__global__ void k_tuple_keys(const TupleVec* tv, const TupleTab* tabs) {
  const TupleVec V = tv[blockIdx.y];
  const TupleTab T = tabs[V.tab];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.n) return;
  for (uint32_t k = 0; k < T.w; k++) T.keys[(uint64_t)(V.comb_off + i) * T.w + k] = V.comp[k][i];
}
__global__ void k_tuple_insert(const TupleVec* tv, const TupleTab* tabs, uint32_t* fail) {
  const TupleVec V = tv[blockIdx.y];
  const TupleTab T = tabs[V.tab];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.n || (V.sel && V.sel[i] == 0)) return;
  const uint32_t g = V.comb_off + i, mask = T.cap - 1;
  uint32_t h = tuple_hash(V, i, T.w, mask);
  for (uint32_t probe = 0; probe < T.cap; probe++, h = (h + 1) & mask) {
    const uint32_t prev = atomicCAS(T.rep + h, MULT_EMPTY, g);
    if (prev == MULT_EMPTY || tuple_eq(V, i, T.keys + (uint64_t)prev * T.w, T.w)) {
      atomicMin(T.first + h, g);
      return;
    }
  }
  atomicOr(fail, 2u);
}
__global__ void k_tuple_count(const TupleVec* sv, const TupleTab* tabs, uint32_t* missing) {
  const TupleVec V = sv[blockIdx.y];
  const TupleTab T = tabs[V.tab];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.n) return;
  const uint32_t sel = V.sel ? V.sel[i] : MONT_ONE;
  if (sel == 0) return;
  const uint32_t mask = T.cap - 1;
  uint32_t h = tuple_hash(V, i, T.w, mask);
  for (uint32_t probe = 0; probe < T.cap; probe++, h = (h + 1) & mask) {
    const uint32_t r = T.rep[h];
    if (r == MULT_EMPTY) break;
    if (tuple_eq(V, i, T.keys + (uint64_t)r * T.w, T.w)) {
      atomicAdd(T.weight + h, (unsigned long long)from_mont(sel));
      return;
    }
  }
  atomicOr(missing, 1u);
}
__global__ void k_tuple_write(const TupleVec* tv, const TupleTab* tabs) {
  const TupleVec V = tv[blockIdx.y];
  const TupleTab T = tabs[V.tab];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.n) return;
  uint32_t m = 0;
  const uint32_t sel = V.sel ? V.sel[i] : MONT_ONE;
  if (sel != 0) {
    const uint32_t g = V.comb_off + i, mask = T.cap - 1;
    uint32_t h = tuple_hash(V, i, T.w, mask);
    for (uint32_t probe = 0; probe < T.cap; probe++, h = (h + 1) & mask) {
      const uint32_t r = T.rep[h];
      if (r == MULT_EMPTY) break;
      if (tuple_eq(V, i, T.keys + (uint64_t)r * T.w, T.w)) {
        if (T.first[h] == g) m = mul(to_mont((uint32_t)(T.weight[h] % P)), V.sel ? inv(sel) : MONT_ONE);
        break;
      }
    }
  }
  V.out[i] = m;
}

// Values of a base-field expression on every row (for lookup tables that are
// not plain columns).
struct EvalJob { XProgram p; const uint32_t* const* lanes; uint32_t* out; int logn; };
__global__ void k_eval_base(const EvalJob* jobs, const E6* coins) {
  extern __shared__ uint32_t regs[];
  const EvalJob& J = jobs[blockIdx.y];
  const uint32_t n = 1u << J.logn;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t* const* lanes = J.lanes;
  auto lane = [&](uint32_t l, uint32_t row) -> uint32_t { return lanes[l][row]; };
  J.out[j] = x_eval(J.p, coins, regs + threadIdx.x, blockDim.x, j, n, lane).c[0];
}

// ---------------------------------------------------------------- claimed values
// zp[k] = z^k, k < n.
__global__ void k_e6_powers(const uint32_t* zw, uint32_t ws, uint32_t n, uint32_t* zp) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  E6 z;
#pragma unroll
  for (int w = 0; w < 6; w++) z.c[w] = zw[w];
  E6 v = e6_pow(e6_mul_base(z, ws), k);
  st6(zp, n, k, v);
}

// One block per (lane, point): out = sum_k coef[k] z^k (E6).
struct DotJob { const uint32_t* coef; const uint32_t* zp; uint32_t n; uint32_t out_idx; };
__global__ void k_dot(const DotJob* jobs, uint32_t* out) {
  __shared__ E6 part[256];
  DotJob jb = jobs[blockIdx.x];
  E6 acc = e6_zero();
  for (uint32_t k = threadIdx.x; k < jb.n; k += blockDim.x) {
    uint32_t c = jb.coef[k];
    for (int w = 0; w < 6; w++) acc.c[w] = add(acc.c[w], mul(jb.zp[(uint64_t)w * jb.n + k], c));
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (threadIdx.x < (unsigned)off) part[threadIdx.x] = e6_add(part[threadIdx.x], part[threadIdx.x + off]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int w = 0; w < 6; w++) out[jb.out_idx * 6 + w] = part[0].c[w];
}

// ---------------------------------------------------------------- DEEP
// DQ(x) = sum_s (A_s - sum_{b in s} alpha^i_b P_b(x)) / (z_s - x) on the LDE
// rows r of one class, x = w_4n^bitrev(r) (internal/fri/deep.go:205-266,
// evaluated on the 4n LDE rows instead of the n trace rows and re-encoded:
// DQ has degree < n, so both give the same codeword).
constexpr int DEEP_MAX_POINTS = 4;
struct DeepBundle { const uint32_t* lane0; uint64_t lane_stride; uint32_t ext; uint32_t mask; E6 scale; };
struct DeepJob {
  const DeepBundle* bundles;
  uint32_t n_bundles;
  uint32_t n_points;
  E6 z[DEEP_MAX_POINTS];
  E6 a[DEEP_MAX_POINTS];
  int logn4;            // log2 of the LDE size
  const uint32_t* tw;   // w_4n^j table
  uint32_t* out;        // 6 lanes, lane stride 4n
  const uint32_t* den;  // 1/(z_s - x) from k_deep_den (null: computed here)
};

// The DEEP denominators 1/(z_s - x) of every LDE row r of a class (x =
// w_4n^bitrev(r)), one inversion per row for all its points (Montgomery's
// trick), stored as six lanes per point: den[(6 s + w) 4n + r].  z_s =
// zeta ws[s] with zeta read from its device slot, so the kernel runs as
// soon as zeta is known, beside the claimed values and the host's
// alpha_DEEP transcript.
struct DenJob { uint32_t n_points; uint32_t ws[DEEP_MAX_POINTS]; int logn4; const uint32_t* tw; uint32_t* den; };
__global__ void k_deep_den(const DenJob* jobs, const uint32_t* zeta_w) {
  const DenJob& jb = jobs[blockIdx.y];
  const uint32_t big = 1u << jb.logn4;
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= big) return;
  E6 zeta;
#pragma unroll
  for (int w = 0; w < 6; w++) zeta.c[w] = zeta_w[w];
  const uint32_t x = __ldg(jb.tw + bitrev32(r, jb.logn4));
  const uint32_t np = jb.n_points;
  E6 d[DEEP_MAX_POINTS], pre[DEEP_MAX_POINTS];
  for (uint32_t s = 0; s < np; s++) {
    d[s] = e6_mul_base(zeta, jb.ws[s]);
    d[s].c[0] = sub(d[s].c[0], x);
    pre[s] = s ? e6_mul(pre[s - 1], d[s]) : d[s];
  }
  auto put = [&](uint32_t s, const E6& v) {
#pragma unroll
    for (int w = 0; w < 6; w++) jb.den[(uint64_t)(6 * s + w) * big + r] = v.c[w];
  };
  E6 inv_run = e6_inv(pre[np - 1]);
  for (uint32_t s = np - 1; s > 0; s--) {
    put(s, e6_mul(inv_run, pre[s - 1]));
    inv_run = e6_mul(inv_run, d[s]);
  }
  put(0, inv_run);
}
__global__ void k_deep(const DeepJob* jobs) {
  const DeepJob& jb = jobs[blockIdx.y];
  const uint32_t big = 1u << jb.logn4;
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= big) return;
  E6 acc[DEEP_MAX_POINTS];
  for (uint32_t s = 0; s < jb.n_points; s++) acc[s] = jb.a[s];
  for (uint32_t b = 0; b < jb.n_bundles; b++) {
    DeepBundle bu = jb.bundles[b];
    E6 v;
    if (bu.ext) {
      E6 px;
      for (int w = 0; w < 6; w++) px.c[w] = bu.lane0[w * bu.lane_stride + r];
      v = e6_mul(bu.scale, px);
    } else {
      v = e6_mul_base(bu.scale, bu.lane0[r]);
    }
    for (uint32_t s = 0; s < jb.n_points; s++)
      if (bu.mask >> s & 1) acc[s] = e6_sub(acc[s], v);
  }
  const uint32_t np = jb.n_points;
  if (jb.den) {  // the denominators are precomputed
    E6 dq = e6_zero();
    for (uint32_t s = 0; s < np; s++) {
      E6 is;
#pragma unroll
      for (int w = 0; w < 6; w++) is.c[w] = jb.den[(uint64_t)(6 * s + w) * big + r];
      dq = e6_add(dq, e6_mul(acc[s], is));
    }
    for (int w = 0; w < 6; w++) jb.out[(uint64_t)w * big + r] = dq.c[w];
    return;
  }
  uint32_t x = __ldg(jb.tw + bitrev32(r, jb.logn4));
  // sum_s acc_s / (z_s - x) with one inversion (Montgomery's trick over the
  // points): pre_s = d_0 ... d_s, then 1/d_s = pre_(s-1) / pre_s from the top
  E6 d[DEEP_MAX_POINTS], pre[DEEP_MAX_POINTS];
  for (uint32_t s = 0; s < np; s++) {
    d[s] = jb.z[s];
    d[s].c[0] = sub(d[s].c[0], x);
    pre[s] = s ? e6_mul(pre[s - 1], d[s]) : d[s];
  }
  E6 dq = e6_zero();
  if (np) {
    E6 inv_run = e6_inv(pre[np - 1]);  // 1 / (d_0 ... d_(np-1))
    for (uint32_t s = np - 1; s > 0; s--) {
      dq = e6_add(dq, e6_mul(acc[s], e6_mul(inv_run, pre[s - 1])));
      inv_run = e6_mul(inv_run, d[s]);
    }
    dq = e6_add(dq, e6_mul(acc[0], inv_run));
  }
  for (int w = 0; w < 6; w++) jb.out[(uint64_t)w * big + r] = dq.c[w];
}

// ---------------------------------------------------------------- FRI
// running += sum_t gamma_t * level_t (6 lanes each, lane stride n), the
// levels entering FRI at this round in level order.
// gamma: device words (the first six words of the challenge's digest).
struct AxpyTerm { const uint32_t* lvl; const uint32_t* gamma; };
__device__ __forceinline__ E6 ld_e6w(const uint32_t* w) {
  E6 r;
#pragma unroll
  for (int k = 0; k < 6; k++) r.c[k] = w[k];
  return r;
}
__global__ void k_axpy_e6(uint32_t* run, uint64_t n, const AxpyTerm* terms, uint32_t n_terms) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  E6 a = ld6(run, n, i);
  for (uint32_t t = 0; t < n_terms; t++) a = e6_add(a, e6_mul(ld6(terms[t].lvl, n, i), ld_e6w(terms[t].gamma)));
  st6(run, n, i, a);
}

// next[i] = (p+q)/2 + alpha (p-q)/(2 x_i), x_i^-1 = w_n^-bitrev(i, n/2)
// (internal/fri/fri.go:1113-1118,1177-1198).  tw: w_n^j table.
// alpha: device words (the first six words of a challenge digest).
__global__ void k_fold(const uint32_t* layer, uint64_t n, const uint32_t* alpha_w, const uint32_t* tw, uint32_t inv2,
                       uint32_t* next) {
  const uint64_t half = n / 2;
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= half) return;
  E6 alpha;
#pragma unroll
  for (int w = 0; w < 6; w++) alpha.c[w] = __ldg(alpha_w + w);
  int lg = 0;
  while ((1ull << lg) < half) lg++;
  uint32_t e = bitrev32((uint32_t)i, lg);
  uint32_t xinv = __ldg(tw + ((n - e) & (n - 1)));
  E6 p = ld6(layer, n, 2 * i), q = ld6(layer, n, 2 * i + 1);
  E6 s = e6_mul_base(e6_add(p, q), inv2);
  E6 d = e6_mul(e6_mul_base(e6_mul_base(e6_sub(p, q), inv2), xinv), alpha);
  st6(next, half, i, e6_add(s, d));
}

// The last FRI rounds in one block: for each round j, the fold of layer j
// with challenge j (as k_fold), the levels that enter at j + 1 (as
// k_axpy_e6), then, unless j is the last round, layer j + 1's commitment —
// pair leaves (one permutation each, as k_hash_leaves), the tree level by
// level — and challenge j + 1 from its root (as k_fs_challenge).  These
// layers are small (at most a few thousand leaves), so their launches were
// latency bound: one block runs them back to back with barriers instead,
// every value written where the per-round launches write it.  Six lanes per
// permutation, five permutations per warp.
struct FriRound {
  const uint32_t* cur;     // layer j: 6 lanes of n words (bit-reversed rows)
  uint32_t* next;          // layer j + 1: 6 lanes of n / 2 words
  const uint32_t* tw;      // w_n^k, k < n
  uint32_t* nodes;         // layer j + 1's tree (2 leaves digests, 1-indexed); null after the last fold
  uint64_t n;              // rows of layer j
  uint32_t log_leaves;     // of that tree
  uint32_t pre_off, pre_len;      // challenge j + 1's name elements in `pre`
  uint32_t term_first, term_count;  // levels added to layer j + 1
};
__global__ void __launch_bounds__(1024) k_fri_tail(const FriRound* rounds, uint32_t n_rounds, uint32_t j0,
                                                   const AxpyTerm* terms, const uint32_t* pre, uint32_t* chal,
                                                   uint32_t inv2) {
  __shared__ uint32_t keys[144];
  __shared__ uint32_t msg[64];
  p2_load_full_keys(keys);  // ends with a barrier
  P2Lane L;
  L.init();
  const uint32_t warps = blockDim.x >> 5, per = warps * P2_GROUPS_PER_WARP;
  const uint32_t slot = (threadIdx.x >> 5) * P2_GROUPS_PER_WARP + (uint32_t)L.base / 6;
  for (uint32_t r = 0; r < n_rounds; r++) {
    const FriRound R = rounds[r];
    const uint32_t j = j0 + r;
    const uint64_t half = R.n / 2;
    // fold
    {
      E6 alpha;
#pragma unroll
      for (int w = 0; w < 6; w++) alpha.c[w] = chal[8 * (size_t)j + w];
      int lg = 0;
      while ((1ull << lg) < half) lg++;
      for (uint64_t i = threadIdx.x; i < half; i += blockDim.x) {
        const uint32_t e = bitrev32((uint32_t)i, lg);
        const uint32_t xinv = __ldg(R.tw + ((R.n - e) & (R.n - 1)));
        const E6 p = ld6(R.cur, R.n, 2 * i), q = ld6(R.cur, R.n, 2 * i + 1);
        const E6 sm = e6_mul_base(e6_add(p, q), inv2);
        const E6 d = e6_mul(e6_mul_base(e6_mul_base(e6_sub(p, q), inv2), xinv), alpha);
        E6 v = e6_add(sm, d);
        for (uint32_t t = 0; t < R.term_count; t++) {
          const AxpyTerm T = terms[R.term_first + t];
          v = e6_add(v, e6_mul(ld6(T.lvl, half, i), ld_e6w(T.gamma)));
        }
        st6(R.next, half, i, v);
      }
    }
    __syncthreads();
    if (!R.nodes) break;
    // leaves of layer j + 1: Sponge(LEAF, 0, 2, row 2k, row 2k + 1), 15 elements
    const uint32_t nl = 1u << R.log_leaves;
    {
      LeafGroup g;
      g.base = nullptr;
      g.ext = R.next;
      g.stride = half;
      g.nb = 0;
      g.ne = 1;
      g.n_leaves = nl;
      g.out = R.nodes + (size_t)8 * nl;
      const uint32_t h0 = to_mont(LEAF_TAG), h1 = to_mont(0), h2 = to_mont(2);
      for (uint32_t k0 = 0; k0 < nl; k0 += per) {
        const uint32_t k = k0 + slot;
        const bool active = L.lane < 30 && k < nl;
        uint32_t x[4] = {0, 0, 0, 0};
        if (active && L.idx < 4) {
#pragma unroll
          for (uint32_t i = 0; i < 4; i++) {
            const uint32_t e = 4 * L.idx + i;
            if (e < 15) x[i] = leaf_elem(g, e, k, h0, h1, h2);
          }
        }
        p2c_permute(x, L, keys);
        if (active && L.idx < 2) {
          uint32_t* o = g.out + (size_t)k * 8 + 4 * L.idx;
#pragma unroll
          for (int i = 0; i < 4; i++) o[i] = x[i];
        }
      }
    }
    __syncthreads();
    for (uint32_t w = nl >> 1; w >= 1; w >>= 1) {
      for (uint32_t i0 = 0; i0 < w; i0 += per) {
        const uint32_t i = i0 + slot;
        merkle_node(R.nodes, (uint64_t)w + i, L, keys, L.lane < 30 && i < w);
      }
      __syncthreads();
    }
    // challenge j + 1 = sponge(name elements || challenge j || root)
    const uint32_t total = R.pre_len + 16;
    for (uint32_t i = threadIdx.x; i < total; i += blockDim.x)
      msg[i] = i < R.pre_len ? pre[R.pre_off + i] : (i < R.pre_len + 8 ? chal[8 * (size_t)j + (i - R.pre_len)]
                                                                          : R.nodes[8 + (i - R.pre_len - 8)]);
    __syncthreads();
    if (threadIdx.x < 32) {
      uint32_t x[4] = {0, 0, 0, 0};
      for (uint32_t b = 0; b < total; b += 16) {
        const uint32_t len = min(16u, total - b);
        if (L.idx < 4)
#pragma unroll
          for (int k = 0; k < 4; k++)
            if (4 * (uint32_t)L.idx + k < len) x[k] = msg[b + 4 * L.idx + k];
        p2c_permute(x, L, keys);
      }
      if (L.lane < 2)
#pragma unroll
        for (int k = 0; k < 4; k++) chal[8 * (size_t)(j + 1) + 4 * L.lane + k] = x[k];
    }
    __syncthreads();
  }
}

// One Fiat-Shamir challenge on the device, for challenges whose bindings are
// already in device memory (the FRI layer roots): digest = state[0..8) of
// the width-24 sponge (rate 16, overwrite, no padding) over
// pre[0..n_pre) || prev[0..8) || bind[0..8), as Transcript::compute on the
// host (internal/fiat-shamir/transcript.go:221-315).  One warp, six lanes
// per permutation; `out` gets 8 words.
__global__ void k_fs_challenge(const uint32_t* pre, uint32_t n_pre, const uint32_t* prev, const uint32_t* bind,
                               uint32_t* out) {
  __shared__ uint32_t keys[144];
  __shared__ uint32_t msg[64];
  const uint32_t total = n_pre + 16;  // n_pre <= 48, checked by the host
  for (uint32_t i = threadIdx.x; i < total; i += blockDim.x)
    msg[i] = i < n_pre ? pre[i] : (i < n_pre + 8 ? prev[i - n_pre] : bind[i - n_pre - 8]);
  p2_load_full_keys(keys);  // ends with a barrier
  P2Lane L;
  L.init();
  uint32_t x[4] = {0, 0, 0, 0};
  for (uint32_t b = 0; b < total; b += 16) {
    const uint32_t len = min(16u, total - b);  // words 0..len of the state are overwritten
    if (L.idx < 4)
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (4 * (uint32_t)L.idx + k < len) x[k] = msg[b + 4 * L.idx + k];
    p2c_permute(x, L, keys);
  }
  if (L.lane < 2)
#pragma unroll
    for (int k = 0; k < 4; k++) out[4 * L.lane + k] = x[k];
}

// A chain of Fiat-Shamir challenges on the device, computed in order:
// challenge i hashes msg[moff, moff + total) as k_fs_challenge does and
// writes its 8 digest words to `out`.  The message words come from segments
// — host constants uploaded with the descriptors (names' elements, known
// bindings) and words already in device memory (roots, exposed values, the
// digest of a challenge computed by an earlier launch) — all read up front,
// one segment per thread at a time; a digest that the next challenge of the
// same chain hashes is forwarded from registers to msg[fwd] instead.  One
// warp, six lanes per permutation; the chain's messages hold at most
// FS_MAX_MSG words (checked by the host).
constexpr uint32_t FS_MAX_MSG = 4096;
struct FsSeg { const uint32_t* src; uint32_t len, off; };
struct FsChal { uint32_t moff, total; uint32_t* out; int32_t fwd; };
__global__ void __launch_bounds__(32) k_fs_chain(const FsChal* chals, uint32_t n_chals, const FsSeg* segs,
                                                 uint32_t n_segs) {
  __shared__ uint32_t keys[144];
  __shared__ uint32_t msg[FS_MAX_MSG];
  for (uint32_t s = threadIdx.x; s < n_segs; s += blockDim.x) {
    const FsSeg sg = segs[s];
    for (uint32_t k = 0; k < sg.len; k++) msg[sg.off + k] = sg.src[k];
  }
  p2_load_full_keys(keys);  // ends with a barrier
  P2Lane L;
  L.init();
  for (uint32_t i = 0; i < n_chals; i++) {
    const FsChal ch = chals[i];
    uint32_t x[4] = {0, 0, 0, 0};
    for (uint32_t b = 0; b < ch.total; b += 16) {
      const uint32_t len = min(16u, ch.total - b);  // words 0..len of the state are overwritten
      if (L.idx < 4)
#pragma unroll
        for (int k = 0; k < 4; k++)
          if (4 * (uint32_t)L.idx + k < len) x[k] = msg[ch.moff + b + 4 * L.idx + k];
      p2c_permute(x, L, keys);
    }
    if (L.lane < 2)
#pragma unroll
      for (int k = 0; k < 4; k++) {
        ch.out[4 * L.lane + k] = x[k];
        if (ch.fwd >= 0) msg[ch.fwd + 4 * L.lane + k] = x[k];
      }
    __syncwarp();
  }
}

// The challenge table of the step and quotient kernels: the round coins (the
// first six words of each digest slot, slot stride 8), then the exposed
// values times ninv[e] (1/n of the producing module; 0 while entry e is not
// produced yet, which zeroes it) and the exposed values themselves.
__global__ void k_coins_assemble(const uint32_t* slots, uint32_t n_coins, const uint32_t* exposed,
                                 const uint32_t* ninv, uint32_t n_exp, uint32_t* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nc = 6 * n_coins, ne = 6 * n_exp;
  if (i < nc) {
    out[i] = slots[8 * (i / 6) + i % 6];
  } else if (i < nc + ne) {
    const uint32_t k = i - nc, f = ninv[k / 6];
    out[i] = f ? mul(exposed[k], f) : 0u;
  } else if (i < nc + 2 * ne) {
    const uint32_t k = i - nc - ne;
    out[i] = ninv[k / 6] ? exposed[k] : 0u;
  }
}

// ---------------------------------------------------------------- openings
// Montgomery words -> canonical values as big-endian bytes (the proof
// encoding), in place.
__global__ void k_proof_words(uint32_t* x, uint64_t n) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) x[i] = __byte_perm(from_mont(x[i]), 0, 0x0123);
}

// Row pairs: for every query q and source, the rows lo and lo + 1 of each
// lane, lo = (s_q >> shift) & ~1: row lo of every lane, then row lo + 1, at
// out[q * per_q + off + h * n_lanes + lane] (the order the proof lists them).
struct RowSrc { const uint32_t* lane0; uint64_t lane_stride; uint32_t n_lanes; uint32_t shift; uint64_t off; };
__global__ void k_gather_rows(const RowSrc* srcs, uint32_t n_src, const uint32_t* pos, uint32_t nq, uint64_t per_q,
                              uint32_t* out) {
  const uint32_t q = blockIdx.y;
  const RowSrc s = srcs[blockIdx.z];
  const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq || l >= s.n_lanes) return;
  uint32_t lo = (pos[q] >> s.shift) & ~1u;
  const uint32_t* p = s.lane0 + l * s.lane_stride;
  out[q * per_q + s.off + l] = p[lo];
  out[q * per_q + s.off + s.n_lanes + l] = p[lo + 1];
}

// Merkle paths: siblings of leaf idx = ((s_q >> shift) >> 1), leaf level
// first, then the injection leaves inj_t[idx >> d_t].
struct PathSrc {
  const uint32_t* nodes;
  const uint32_t* const* inj;
  const uint32_t* inj_shift;  // d_t = log2(n_leaves / width_t)
  uint32_t log_leaves;
  uint32_t n_inj;
  uint32_t shift;
  uint64_t off;
};
__global__ void k_gather_paths(const PathSrc* srcs, const uint32_t* pos, uint32_t nq, uint64_t per_q, uint32_t* out) {
  const uint32_t q = blockIdx.y;
  const PathSrc s = srcs[blockIdx.z];
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq || t >= s.log_leaves + s.n_inj) return;
  uint32_t idx = (pos[q] >> s.shift) >> 1;
  uint32_t* o = out + q * per_q + s.off + (uint64_t)t * 8;
  const uint32_t* src;
  if (t < s.log_leaves) {
    uint64_t node = (((uint64_t)1 << s.log_leaves) + idx) >> t;
    src = s.nodes + (node ^ 1) * 8;
  } else {
    uint32_t k = t - s.log_leaves;
    src = s.inj[k] + (uint64_t)(idx >> s.inj_shift[k]) * 8;
  }
  for (int w = 0; w < 8; w++) o[w] = src[w];
}

// Per-query proof sections.  Every query's part of a section has the same
// layout, described once per section by a word map: code >> 30 = 0 copies
// gathered word (code & 0x3fffffff) of the query, 1 is constant word
// consts[code & ..], 2 is a position word of pos_ops[code & ..] (the query's
// row or leaf index at some layer).  Output: big-endian words, query k of
// section s at out + s.out_off + k * s.q_words.
struct PosOp { uint32_t shift, leaf; };
struct SectionSrc { uint64_t map_off, out_off; uint32_t q_words; };
constexpr uint32_t SEC_COPY = 0u, SEC_CONST = 1u, SEC_POS = 2u;
__global__ void k_assemble(const SectionSrc* secs, const uint32_t* map, const uint32_t* consts, const PosOp* pops,
                           const uint32_t* pos, const uint32_t* gathered, uint64_t per_q, uint32_t nq, uint32_t* out) {
  const SectionSrc sc = secs[blockIdx.z];
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (j >= sc.q_words || k >= nq) return;
  const uint32_t code = map[sc.map_off + j], kind = code >> 30, idx = code & 0x3fffffffu;
  uint32_t w;
  if (kind == SEC_COPY) {
    w = gathered[(uint64_t)k * per_q + idx];  // already big-endian (k_proof_words)
  } else {
    uint32_t v;
    if (kind == SEC_CONST) {
      v = consts[idx];
    } else {
      const PosOp op = pops[idx];
      v = pos[k] >> op.shift;
      if (op.leaf) v = (v & ~1u) >> 1;
    }
    w = __byte_perm(v, 0, 0x0123);
  }
  out[sc.out_off + (uint64_t)k * sc.q_words + j] = w;
}

}  // namespace lg
