// Shared-memory transforms of 2^4 .. 2^14 points with 16 elements per thread
// in registers.  The stages run in passes of up to four: a thread loads the
// 16 elements whose indices differ in the pass's four "local" bits, runs the
// pass's radix-2 stages in registers, and writes them back — one shared-memory
// round trip and one barrier per four stages instead of per stage.
//
// Shared memory is addressed with one pad word per 16 (pad16) so that the
// 16-element groups of a warp fall into distinct banks in every pass.
#pragma once
#include <type_traits>
#include <utility>

#include "field.cuh"

namespace lg {

__device__ __forceinline__ uint32_t pad16(uint32_t i) { return i + (i >> 4); }

// index of element r (0..15) of group t when the local bits are [lo, lo+4)
__device__ __forceinline__ uint32_t grp_index(uint32_t t, uint32_t r, int lo) {
  return ((t >> lo) << (lo + 4)) | (r << lo) | (t & ((1u << lo) - 1));
}

// Pass plan.  DIF: the first pass takes the top logn mod 4 stages (or 4) with
// local bits [logn-4, logn); then four stages per pass.  DIT mirrors it from
// the bottom.
LG_HD constexpr int pass_count(int logn) {
  return (logn - ((logn & 3) ? (logn & 3) : 4)) / 4 + 1;
}
template <bool DIF>
LG_HD constexpr void pass_plan(int p, int logn, int& lo, int& s_lo, int& s_hi) {
  const int rem = (logn & 3) ? (logn & 3) : 4;
  if (DIF) {
    if (p == 0) { lo = logn - 4; s_hi = logn - 1; s_lo = logn - rem; }
    else { s_hi = logn - rem - 4 * (p - 1) - 1; s_lo = s_hi - 3; lo = s_lo; }
  } else {
    const int np = pass_count(logn);
    if (p < np - 1) { s_lo = 4 * p; s_hi = s_lo + 3; lo = s_lo; }
    else { s_lo = 4 * p; s_hi = logn - 1; lo = logn - 4; }
  }
}

// Twiddle tables laid out pass by pass.  Stage s of a pass with local bits
// [lo, lo + 4) multiplies by w_{2^(s+1)}^j, j = (t mod 2^lo) + r 2^lo for the
// thread's group t and the register pair r < 2^(s-lo): for each t mod 2^lo
// those 2^(s-lo) values sit next to each other, so a thread reads a stage's
// twiddles with one or two vector loads (one table entry per (t mod 2^lo, r):
// 2^s words per stage, each stage's block rounded up to 8 words).  Four
// regions: DIF forward, DIF inverse, DIT forward, DIT inverse.
//
// The twiddles are canonical values with their Shoup companions (field.cuh
// mulc): the tw16_words(logn) canonical words, then as many companions at
// the same offsets.  A product by a fixed twiddle then takes one high and two
// low 32-bit multiplies instead of Montgomery's two wide ones (on B200 about
// 1.5 x the products per clock, 1.4-1.6 x the butterflies).
LG_HD constexpr uint32_t tw16_round8(uint32_t w) { return (w + 7u) & ~7u; }
LG_HD constexpr uint32_t tw16_pass_words(int logn, bool dif, int p) {
  int lo = 0, s_lo = 0, s_hi = 0;
  if (dif) pass_plan<true>(p, logn, lo, s_lo, s_hi);
  else pass_plan<false>(p, logn, lo, s_lo, s_hi);
  uint32_t w = 0;
  for (int s = s_lo; s <= s_hi; s++) w += tw16_round8(1u << s);
  return w;
}
LG_HD constexpr uint32_t tw16_region_words(int logn, bool dif) {
  uint32_t w = 0;
  for (int p = 0; p < pass_count(logn); p++) w += tw16_pass_words(logn, dif, p);
  return w;
}
LG_HD constexpr uint32_t tw16_words(int logn) { return 2 * tw16_region_words(logn, true) + 2 * tw16_region_words(logn, false); }
// offset of pass p's table
LG_HD constexpr uint32_t tw16_pass_offset(int logn, bool dif, bool inverse, int p) {
  uint32_t off = dif ? 0u : 2 * tw16_region_words(logn, true);
  if (inverse) off += tw16_region_words(logn, dif);
  for (int q = 0; q < p; q++) off += tw16_pass_words(logn, dif, q);
  return off;
}
// offset of stage s's block inside its pass's table
LG_HD constexpr uint32_t tw16_stage_offset(int s_lo, int s) {
  uint32_t off = 0;
  for (int q = s_lo; q < s; q++) off += tw16_round8(1u << q);
  return off;
}

// m consecutive words from an m-aligned offset (m = 1, 2, 4, 8)
template <int M> __device__ __forceinline__ void ld_tw(const uint32_t* p, uint32_t* w) {
  if constexpr (M == 1) {
    w[0] = __ldg(p);
  } else if constexpr (M == 2) {
    const uint2 a = __ldg(reinterpret_cast<const uint2*>(p));
    w[0] = a.x; w[1] = a.y;
  } else {
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    if constexpr (M == 8) {
      const uint4 b = __ldg(reinterpret_cast<const uint4*>(p) + 1);
      w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
    }
  }
}

// w_{2^(S+1)}^RL (or its inverse), canonical, with its Shoup companion, as
// compile-time constants: the pass whose local bits are the lowest four
// (lo = 0) has the same twiddles in every thread, j = RL.
template <int S, int RL, bool INV> struct TwConst {
  static constexpr uint32_t order = 2u << S;
  static constexpr uint32_t w = cx_pow(3, (uint64_t)127 << (24 - (S + 1)));  // canonical, order 2^(S+1)
  static constexpr uint32_t value = cx_pow(w, INV ? (order - RL) % order : RL);
  static constexpr uint32_t comp = shoup(value);
};

template <int LS, bool INV, size_t... R>
__device__ __forceinline__ void tw_consts(uint32_t* w, uint32_t* ws, std::index_sequence<R...>) {
  ((w[R] = TwConst<LS, (int)R, INV>::value, ws[R] = TwConst<LS, (int)R, INV>::comp), ...);
}

// Stages s in [s_lo, s_hi] on the 16 registers of group t (local bits
// [lo, lo+4)).  DIF: (u, v) -> (u + v, (u - v) w), stages descending;
// DIT: (u, v) -> (u + v w, u - v w), stages ascending.  w = w_{2^(s+1)}^j,
// j = index mod 2^s; `ptab`: this pass's twiddle table (tw16 layout), its
// companions `comp` words further on.  When lo = 0 the twiddles are
// constants (j = r) and w = 1 (r = 0) costs no product.
template <bool DIF, int LS>
__device__ __forceinline__ void stage16(uint32_t v[16], uint32_t t, int lo, int s_lo, const uint32_t* ptab,
                                        uint32_t comp, bool inverse) {
  constexpr uint32_t m = 1u << LS;
  const int s = lo + LS;
  uint32_t w[m], ws[m];
  if (lo == 0) {
    if (inverse) tw_consts<LS, true>(w, ws, std::make_index_sequence<m>{});
    else tw_consts<LS, false>(w, ws, std::make_index_sequence<m>{});
  } else {
    const uint32_t* at = ptab + tw16_stage_offset(s_lo, s) + (t & ((1u << lo) - 1)) * m;
    ld_tw<m>(at, w);
    ld_tw<m>(at + comp, ws);
  }
#pragma unroll
  for (uint32_t rl = 0; rl < m; rl++) {
    const bool unit = lo == 0 && rl == 0;
#pragma unroll
    for (uint32_t rh = 0; rh < 16; rh += 2 * m) {
      uint32_t& a = v[rh + rl];
      uint32_t& b = v[rh + rl + m];
      if (DIF) {
        uint32_t u = a, x = b;
        a = add(u, x);
        b = unit ? sub(u, x) : mulc(sub_lazy(u, x), w[rl], ws[rl]);
      } else {
        uint32_t u = a, x = unit ? b : mulc(b, w[rl], ws[rl]);
        a = add(u, x);
        b = sub(u, x);
      }
    }
  }
}
template <bool DIF>
__device__ __forceinline__ void pass16(uint32_t v[16], uint32_t t, int lo, int s_lo, int s_hi, const uint32_t* ptab,
                                       uint32_t comp, bool inverse) {
  auto one = [&](auto LSC) {
    constexpr int LS = decltype(LSC)::value;
    const int s = lo + LS;
    if (s >= s_lo && s <= s_hi) stage16<DIF, LS>(v, t, lo, s_lo, ptab, comp, inverse);
  };
  if (DIF) {
    one(std::integral_constant<int, 3>{});
    one(std::integral_constant<int, 2>{});
    one(std::integral_constant<int, 1>{});
    one(std::integral_constant<int, 0>{});
  } else {
    one(std::integral_constant<int, 0>{});
    one(std::integral_constant<int, 1>{});
    one(std::integral_constant<int, 2>{});
    one(std::integral_constant<int, 3>{});
  }
}

struct NoHook {
  __device__ void operator()(uint32_t, const uint32_t*) const {}
};

// Full transform of n = 2^logn >= 16 points; `tw`: the size's radix-16
// twiddle tables (tw16 layout, Ctx::twiddles16).  Pass 0 takes its inputs from
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
  const uint32_t comp = tw16_words(logn);
#pragma unroll
  for (int p = 0; p < np; p++) {
    int lo = 0, s_lo = 0, s_hi = 0;
    pass_plan<DIF>(p, logn, lo, s_lo, s_hi);
    const uint32_t* ptab = tw + tw16_pass_offset(logn, DIF, inverse, p);
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
      pass16<DIF>(v, t, lo, s_lo, s_hi, ptab, comp, inverse);
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
