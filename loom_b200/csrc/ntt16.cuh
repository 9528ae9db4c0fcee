// Shared-memory transforms of 2^4 .. 2^14 points with 16 elements per thread
// in registers.  The stages run in passes of up to four: a thread loads the
// 16 elements whose indices differ in the pass's four "local" bits, runs the
// pass's radix-2 stages in registers, and writes them back — one shared-memory
// round trip and one barrier per four stages instead of per stage.
//
// Shared memory is addressed with one pad word per 16 (pad16) so that the
// 16-element groups of a warp fall into distinct banks in every pass.
#pragma once
#include "field.cuh"

namespace lg {

__device__ __forceinline__ uint32_t pad16(uint32_t i) { return i + (i >> 4); }

// index of element r (0..15) of group t when the local bits are [lo, lo+4)
__device__ __forceinline__ uint32_t grp_index(uint32_t t, uint32_t r, int lo) {
  return ((t >> lo) << (lo + 4)) | (r << lo) | (t & ((1u << lo) - 1));
}

__device__ __forceinline__ uint32_t twid(const uint32_t* tw, uint32_t e, uint32_t mask, bool inverse) {
  return __ldg(tw + (inverse ? ((0u - e) & mask) : e));
}

// Stages s in [s_lo, s_hi] on the 16 registers of group t (local bits
// [lo, lo+4)).  DIF: (u, v) -> (u + v, (u - v) w), stages descending;
// DIT: (u, v) -> (u + v w, u - v w), stages ascending.  w = w_{2^(s+1)}^j,
// j = index mod 2^s.
template <bool DIF>
__device__ __forceinline__ void pass16(uint32_t v[16], uint32_t t, int lo, int s_lo, int s_hi, int logn,
                                       const uint32_t* tw, bool inverse) {
  const uint32_t mask = (1u << logn) - 1;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int ls = DIF ? 3 - k : k;  // local bit of this stage
    const int s = lo + ls;
    if (s < s_lo || s > s_hi) continue;
    const uint32_t m = 1u << ls;
    // twiddle depends on the index bits below s: thread bits below lo and local bits below ls
#pragma unroll
    for (uint32_t rl = 0; rl < m; rl++) {
      const uint32_t i0 = grp_index(t, rl, lo);
      const uint32_t j = i0 & ((1u << s) - 1);
      const uint32_t w = twid(tw, j << (logn - s - 1), mask, inverse);
#pragma unroll
      for (uint32_t rh = 0; rh < 16; rh += 2 * m) {
        uint32_t& a = v[rh + rl];
        uint32_t& b = v[rh + rl + m];
        if (DIF) {
          uint32_t u = a, x = b;
          a = add(u, x);
          b = mul(sub(u, x), w);
        } else {
          uint32_t u = a, x = mul(b, w);
          a = add(u, x);
          b = sub(u, x);
        }
      }
    }
  }
}

// Pass plan.  DIF: the first pass takes the top logn mod 4 stages (or 4) with
// local bits [logn-4, logn); then four stages per pass.  DIT mirrors it from
// the bottom.  Returns the number of passes.
__device__ __forceinline__ int pass_count(int logn) {
  int rem = logn & 3;
  if (!rem) rem = 4;
  return (logn - rem) / 4 + 1;
}
template <bool DIF>
__device__ __forceinline__ void pass_plan(int p, int logn, int& lo, int& s_lo, int& s_hi) {
  int rem = logn & 3;
  if (!rem) rem = 4;
  if (DIF) {
    if (p == 0) { lo = logn - 4; s_hi = logn - 1; s_lo = logn - rem; }
    else { s_hi = logn - rem - 4 * (p - 1) - 1; s_lo = s_hi - 3; lo = s_lo; }
  } else {
    int np = pass_count(logn);
    if (p < np - 1) { s_lo = 4 * p; s_hi = s_lo + 3; lo = s_lo; }
    else { s_lo = 4 * p; s_hi = logn - 1; lo = logn - 4; }
  }
}

struct NoHook {
  __device__ void operator()(uint32_t, const uint32_t*) const {}
};

// Full transform of n = 2^logn >= 16 points.  Pass 0 takes its inputs from
// `first(t, r, lo)` (a global gather, or a shared-memory read with a scale)
// and shows them to `loaded(t, v)` before its butterflies; every pass but the
// last writes back to S (pad16 layout); the last pass hands its 16 registers
// to `store(t, lo, v)`.
//
// Callers instantiate their kernels per size (logn a compile-time constant
// after inlining), so the pass plan, the index arithmetic and the twiddle
// offsets fold into constants and the pass loop unrolls.
template <bool DIF, class First, class Store, class Loaded = NoHook>
__device__ __forceinline__ void ntt16(uint32_t* S, int logn, const uint32_t* tw, bool inverse, First first,
                                      Store store, Loaded loaded = Loaded()) {
  const uint32_t groups = (1u << logn) >> 4;
  const int np = pass_count(logn);
#pragma unroll
  for (int p = 0; p < np; p++) {
    int lo, s_lo, s_hi;
    pass_plan<DIF>(p, logn, lo, s_lo, s_hi);
    for (uint32_t t = threadIdx.x; t < groups; t += blockDim.x) {
      uint32_t v[16];
      if (p == 0) {
#pragma unroll
        for (uint32_t r = 0; r < 16; r++) v[r] = first(t, r, lo);
        loaded(t, v);
      } else {
#pragma unroll
        for (uint32_t r = 0; r < 16; r++) v[r] = S[pad16(grp_index(t, r, lo))];
      }
      pass16<DIF>(v, t, lo, s_lo, s_hi, logn, tw, inverse);
      if (p == np - 1) {
        store(t, lo, v);
      } else {
#pragma unroll
        for (uint32_t r = 0; r < 16; r++) S[pad16(grp_index(t, r, lo))] = v[r];
      }
    }
    __syncthreads();
  }
}

}  // namespace lg
