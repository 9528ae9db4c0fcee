// Transforms of 2^15 .. 2^22 points: four-step, two passes through a scratch
// buffer.  With n = R C (R = 2^floor(log n / 2), C = 2^ceil(log n / 2)),
// k = k1 + R k2 and j = C j1 + j2:
//   X[C j1 + j2] = sum_k1 w_R^(j1 k1) w_n^(j2 k1) sum_k2 w_C^(j2 k2) x[k1 + R k2].
// Pass A: for a tile of 16 consecutive k1, the length-C transforms over k2
// (the tile's 16 columns are read 64 bytes at a time), times w_n^(j2 k1), into
// scratch[j2 R + k1].  Pass B: for a tile of 16 consecutive j2, the length-R
// transforms over k1 (scratch rows, contiguous), stored in natural order
// (X[j]) or in bit-reversed order (out[bitrev(j)], what reedsolomon.Encode
// produces).  Input scaling x[k] * c0 * t1[k] * t2[(e k) mod m2] covers 1/n
// and the coset shifts.
//
// The 16 sub-transforms of a tile run together in shared memory with the
// radix-16 register passes of ntt16.cuh (16 elements of one column per thread,
// four stages per shared-memory round trip), the columns interleaved: element
// (row, col) at 16 (row + row / 16) + (col ^ (row mod 16)).  The row padding
// keeps the two half-warps of a pass in different banks, the column swizzle
// keeps the row-wise staging of pass B conflict-free.
#pragma once
#include "kernels.cuh"

namespace lg {

constexpr int BIG_TILE = 16;

struct BigNtt {
  const uint32_t* in;
  uint32_t* out;
  uint32_t* scratch;       // n words
  const uint32_t* t1;      // optional table of n words (Montgomery)
  const uint32_t* t2;      // optional: the coset shift w_4n^((e2 k) mod 4n) (set: the w_4n table)
  uint32_t m2_mask, e2;    // t2 index = (e2 * k) & m2_mask
  uint32_t c0;             // constant factor (Montgomery)
  uint32_t c0c, c0s;       // c0 canonical and its Shoup companion (big_ntt sets them)
  int out_bitrev;
};

__device__ __forceinline__ uint32_t tile_addr(uint32_t row, uint32_t col) {
  return ((row + (row >> 4)) << 4) + (col ^ (row & 15u));
}
// words of one tile of 16 columns of 2^logl rows
__host__ __device__ constexpr size_t tile_words(int logl) {
  return (((size_t)1 << logl) + ((size_t)1 << logl) / 16) * 16;
}

// The 16 column transforms of a tile, 2^LOGL rows each (`tw`: the tw16
// tables of 2^LOGL points).  Pass 0 takes its
// inputs from first(col, row) (global memory, or the staged tile), every pass
// but the last writes back to S, the last hands each element to
// store(col, row, value) — or, with STORE16 (DIF only: the last pass's local
// bits are the lowest four), a thread's 16 consecutive rows 16 t .. 16 t + 15
// of one column at once to store(col, t, v).  DIF: natural rows in,
// bit-reversed rows out.
template <bool DIF, int LOGL, bool STORE16 = false, class First, class Store>
__device__ __forceinline__ void ntt16_tile(uint32_t* S, const uint32_t* tw, bool inverse, First first, Store store) {
  static_assert(!STORE16 || DIF, "16-row stores follow the DIF pass plan");
  constexpr uint32_t groups = (1u << LOGL) >> 4;  // per column
  constexpr int np = (LOGL - ((LOGL & 3) ? (LOGL & 3) : 4)) / 4 + 1;
  constexpr uint32_t comp = tw16_words(LOGL);
#pragma unroll
  for (int p = 0; p < np; p++) {
    int lo = 0, s_lo = 0, s_hi = 0;
    pass_plan<DIF>(p, LOGL, lo, s_lo, s_hi);
    const uint32_t* ptab = tw + tw16_pass_offset(LOGL, DIF, inverse, p);
    for (uint32_t u = threadIdx.x; u < groups * BIG_TILE; u += blockDim.x) {
      const uint32_t col = u & (BIG_TILE - 1), t = u >> 4;
      uint32_t v[16];
#pragma unroll
      for (uint32_t r = 0; r < 16; r++) {
        const uint32_t row = grp_index(t, r, lo);
        v[r] = p == 0 ? first(col, row) : S[tile_addr(row, col)];
      }
      pass16<DIF>(v, t, lo, s_lo, s_hi, ptab, comp, inverse);
      if constexpr (STORE16) {
        if (p == np - 1) {
          store(col, t, v);
          continue;
        }
      }
#pragma unroll
      for (uint32_t r = 0; r < 16; r++) {
        const uint32_t row = grp_index(t, r, lo);
        if constexpr (!STORE16) {
          if (p == np - 1) {
            store(col, row, v[r]);
            continue;
          }
        }
        S[tile_addr(row, col)] = v[r];
      }
    }
    __syncthreads();
  }
}

// A product v w^e by a power of a root w of order 2^(11 + k), from two small
// tables that stay in L1: lo[i] = w^i (i < 2^11) and hi[i] = w^(2^11 i), each
// entry a canonical word with its Shoup companion (Ctx::split_powers): two
// Shoup products instead of a table product and a Montgomery product.
constexpr int TW_SPLIT = 11;
__device__ __forceinline__ uint32_t mul_split(uint32_t v, const uint2* tab, uint32_t e) {
  const uint2 a = __ldg(tab + (e & ((1u << TW_SPLIT) - 1))), b = __ldg(tab + (1u << TW_SPLIT) + (e >> TW_SPLIT));
  return mulc(mulc_lazy(v, a.x, a.y), b.x, b.y);
}

// tw_n: w_n split (mul_split layout); t2s: the same for w_4n (the coset
// shifts); tw_c: the tw16 tables of C points.  Block (x, y): tile x of job y.
template <int LOGC>
__global__ void __launch_bounds__(512, 2) k_big_pass_a(const BigNtt* jobs, int logn, int logr, int inverse,
                                                    const uint2* tw_n, const uint2* t2s, const uint32_t* tw_c) {
  extern __shared__ uint32_t S[];
  const BigNtt J = jobs[blockIdx.y];
  const uint32_t R = 1u << logr, n = 1u << logn;
  const uint32_t k1_0 = blockIdx.x * BIG_TILE;
  auto first = [&](uint32_t col, uint32_t k2) {
    const uint32_t k = (k1_0 + col) + R * k2;
    uint32_t v = J.in[k];
    if (J.c0 != MONT_ONE) v = mulc(v, J.c0c, J.c0s);
    if (J.t1) v = mul(v, __ldg(J.t1 + k));
    if (J.t2) v = mul_split(v, t2s, (J.e2 * k) & J.m2_mask);
    return v;
  };
  auto store = [&](uint32_t col, uint32_t p, uint32_t v) {
    const uint32_t j2 = bitrev32(p, LOGC), k1 = k1_0 + col;
    uint32_t e = (uint32_t)(((uint64_t)j2 * k1) & (n - 1));
    if (inverse) e = (n - e) & (n - 1);
    J.scratch[(uint64_t)j2 * R + k1] = mul_split(v, tw_n, e);
  };
  ntt16_tile<true, LOGC>(S, tw_c, inverse != 0, first, store);
}

// Block (x, y): rows [16 x, 16 x + 16) of job y's scratch.
template <int LOGR>
__global__ void __launch_bounds__(512, 2) k_big_pass_b(const BigNtt* jobs, int logc, int inverse,
                                                    const uint32_t* tw_r) {
  extern __shared__ uint32_t S[];
  const BigNtt J = jobs[blockIdx.y];
  constexpr uint32_t R = 1u << LOGR;
  const uint32_t C = 1u << logc;
  const uint32_t j2_0 = blockIdx.x * BIG_TILE;
  // stage the 16 scratch rows (contiguous, coalesced) into the tile, every
  // copy in flight before the first wait
  for (uint32_t idx = threadIdx.x; idx < R * BIG_TILE; idx += blockDim.x) {
    const uint32_t jl = idx / R, k1 = idx % R;
    cp_async4(&S[tile_addr(k1, jl)], J.scratch + (uint64_t)(j2_0 + jl) * R + k1);
  }
  cp_async_wait_all();
  __syncthreads();
  auto first = [&](uint32_t col, uint32_t k1) { return S[tile_addr(k1, col)]; };
  if (J.out_bitrev) {
    // out[bitrev_C(j2) R + q] = X[C bitrev_R(q) + j2]: position q holds
    // j1 = bitrev_R(q); a thread's rows q = 16 t .. 16 t + 15 are 64
    // contiguous bytes of one output row
    auto store = [&](uint32_t col, uint32_t t, const uint32_t* v) {
      uint4* o = reinterpret_cast<uint4*>(J.out + (uint64_t)bitrev32(j2_0 + col, logc) * R + 16 * t);
      o[0] = make_uint4(v[0], v[1], v[2], v[3]);
      o[1] = make_uint4(v[4], v[5], v[6], v[7]);
      o[2] = make_uint4(v[8], v[9], v[10], v[11]);
      o[3] = make_uint4(v[12], v[13], v[14], v[15]);
    };
    ntt16_tile<true, LOGR, true>(S, tw_r, inverse != 0, first, store);
  } else {
    auto store = [&](uint32_t col, uint32_t q, uint32_t v) {
      J.out[(uint64_t)C * bitrev32(q, LOGR) + j2_0 + col] = v;
    };
    ntt16_tile<true, LOGR>(S, tw_r, inverse != 0, first, store);
  }
}

// Calls f(std::integral_constant<int, L>{}) for the sub-transform sizes of
// the four-step path, 2^7 .. 2^11 rows.
template <class F> inline void with_tile_size(int logl, F&& f) {
  switch (logl) {
    case 7: f(std::integral_constant<int, 7>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 9: f(std::integral_constant<int, 9>{}); break;
    case 10: f(std::integral_constant<int, 10>{}); break;
    case 11: f(std::integral_constant<int, 11>{}); break;
    default: break;
  }
}

}  // namespace lg
