// Transforms of 2^15 .. 2^22 points: four-step, two passes through a scratch
// buffer.  With n = R C (R = 2^floor(log n / 2), C = 2^ceil(log n / 2)),
// k = k1 + R k2 and j = C j1 + j2:
//   X[C j1 + j2] = sum_k1 w_R^(j1 k1) w_n^(j2 k1) sum_k2 w_C^(j2 k2) x[k1 + R k2].
// Pass A: for a tile of TILE consecutive k1, the length-C transforms over k2
// (rows of the input are contiguous in k1), times w_n^(j2 k1), into
// scratch[j2 R + k1].  Pass B: for a tile of TILE consecutive j2, the
// length-R transforms over k1, stored in natural order (X[j]) or in
// bit-reversed order (out[bitrev(j)], what reedsolomon.Encode produces).
// Input scaling x[k] * c0 * t1[k] * t2[(e k) mod m2] covers 1/n and the
// coset shifts.  All sub-transforms run in shared memory.
#pragma once
#include "kernels.cuh"

namespace lg {

constexpr int BIG_TILE = 16;

struct BigNtt {
  const uint32_t* in;
  uint32_t* out;
  uint32_t* scratch;       // n words
  const uint32_t* t1;      // optional table of n words
  const uint32_t* t2;      // optional table of m2 words (a power of two)
  uint32_t m2_mask, e2;    // t2 index = (e2 * k) & m2_mask
  uint32_t c0;             // constant factor (Montgomery)
  int out_bitrev;
};

// Radix-2 DIF over `len` = 2^lg rows of a [len][TILE] shared array (all TILE
// columns at once); position p ends up holding output index bitrev(p).
__device__ void smem_dif_cols(uint32_t* S, int lg, const uint32_t* tw_len, bool inverse) {
  const uint32_t len = 1u << lg, mask = len - 1;
  for (int s = lg; s >= 1; s--) {
    const uint32_t half = 1u << (s - 1);
    for (uint32_t b = threadIdx.x; b < (len / 2) * BIG_TILE; b += blockDim.x) {
      uint32_t kl = b % BIG_TILE, p = b / BIG_TILE;
      uint32_t jj = p & (half - 1);
      uint32_t i0 = ((p >> (s - 1)) << s) | jj, i1 = i0 + half;
      uint32_t w = tw_at(tw_len, jj << (lg - s), mask, inverse);
      uint32_t u = S[i0 * BIG_TILE + kl], v = S[i1 * BIG_TILE + kl];
      S[i0 * BIG_TILE + kl] = add(u, v);
      S[i1 * BIG_TILE + kl] = mul(sub(u, v), w);
    }
    __syncthreads();
  }
}

// tw_n / tw_c / tw_r: tables of w_n^j, w_C^j, w_R^j.
__global__ void k_big_pass_a(const BigNtt* jobs, int logn, int logr, int logc, int inverse, const uint32_t* tw_n,
                             const uint32_t* tw_c) {
  extern __shared__ uint32_t S[];
  const BigNtt J = jobs[blockIdx.y];
  const uint32_t R = 1u << logr, C = 1u << logc, n = 1u << logn;
  const uint32_t k1_0 = blockIdx.x * BIG_TILE;
  for (uint32_t idx = threadIdx.x; idx < C * BIG_TILE; idx += blockDim.x) {
    uint32_t k2 = idx / BIG_TILE, kl = idx % BIG_TILE;
    uint32_t k = (k1_0 + kl) + R * k2;
    uint32_t v = J.in[k];
    if (J.c0 != MONT_ONE) v = mul(v, J.c0);
    if (J.t1) v = mul(v, __ldg(J.t1 + k));
    if (J.t2) v = mul(v, __ldg(J.t2 + ((J.e2 * k) & J.m2_mask)));
    S[k2 * BIG_TILE + kl] = v;
  }
  __syncthreads();
  smem_dif_cols(S, logc, tw_c, inverse != 0);
  for (uint32_t idx = threadIdx.x; idx < C * BIG_TILE; idx += blockDim.x) {
    uint32_t p = idx / BIG_TILE, kl = idx % BIG_TILE;
    uint32_t j2 = bitrev32(p, logc), k1 = k1_0 + kl;
    uint32_t e = (uint32_t)(((uint64_t)j2 * k1) & (n - 1));
    J.scratch[(uint64_t)j2 * R + k1] = mul(S[p * BIG_TILE + kl], tw_at(tw_n, e, n - 1, inverse != 0));
  }
}

__global__ void k_big_pass_b(const BigNtt* jobs, int logr, int logc, int inverse, const uint32_t* tw_r) {
  extern __shared__ uint32_t S[];
  const BigNtt J = jobs[blockIdx.y];
  const uint32_t R = 1u << logr, C = 1u << logc;
  const uint32_t j2_0 = blockIdx.x * BIG_TILE;
  for (uint32_t idx = threadIdx.x; idx < R * BIG_TILE; idx += blockDim.x) {
    uint32_t jl = idx / R, k1 = idx % R;
    S[k1 * BIG_TILE + jl] = J.scratch[(uint64_t)(j2_0 + jl) * R + k1];
  }
  __syncthreads();
  smem_dif_cols(S, logr, tw_r, inverse != 0);
  if (J.out_bitrev) {
    // out[bitrev_C(j2) R + bitrev_R(j1)] = X[C j1 + j2], and position q holds j1 = bitrev_R(q)
    for (uint32_t idx = threadIdx.x; idx < R * BIG_TILE; idx += blockDim.x) {
      uint32_t jl = idx / R, q = idx % R;
      J.out[(uint64_t)bitrev32(j2_0 + jl, logc) * R + q] = S[q * BIG_TILE + jl];
    }
  } else {
    for (uint32_t idx = threadIdx.x; idx < R * BIG_TILE; idx += blockDim.x) {
      uint32_t q = idx / BIG_TILE, jl = idx % BIG_TILE;
      J.out[(uint64_t)C * bitrev32(q, logr) + j2_0 + jl] = S[q * BIG_TILE + jl];
    }
  }
}

}  // namespace lg
