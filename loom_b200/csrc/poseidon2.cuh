// Poseidon2 over KoalaBear, width 24: initial external layer, 3 full rounds,
// 21 partial rounds (S-box on lane 0), 3 full rounds, S-box x^3
// (recursion/p2_air.go:206-300).  External layer circ(2 M4, M4, ...) with
// gnark-crypto's addition chain for M4 (recursion/p2_air.go:80-104);
// internal layer 1.1^T + diag (recursion/p2_air.go:107-117).
//
// The same code serves the kernels (state in registers, keys in constant
// memory) and the host transcript.
#pragma once
#include "field.cuh"
#include "p2_constants.h"

namespace lg {

static const uint32_t P2_FULL_RK_H[6][24] = LG_P2_FULL_RK_INIT;
static const uint32_t P2_PARTIAL_RK_H[21] = LG_P2_PARTIAL_RK_INIT;
static const uint32_t P2_DIAG_H[24] = LG_P2_DIAG_INIT;
#ifdef __CUDACC__
__constant__ uint32_t P2_FULL_RK_D[6][24] = LG_P2_FULL_RK_INIT;
__constant__ uint32_t P2_PARTIAL_RK_D[21] = LG_P2_PARTIAL_RK_INIT;
__constant__ uint32_t P2_DIAG_D[24] = LG_P2_DIAG_INIT;
#endif

#ifdef __CUDA_ARCH__
#define LG_P2_FULL_RK P2_FULL_RK_D
#define LG_P2_PARTIAL_RK P2_PARTIAL_RK_D
#define LG_P2_DIAG P2_DIAG_D
#else
#define LG_P2_FULL_RK P2_FULL_RK_H
#define LG_P2_PARTIAL_RK P2_PARTIAL_RK_H
#define LG_P2_DIAG P2_DIAG_H
#endif

LG_HD void p2_m4(uint32_t& x0, uint32_t& x1, uint32_t& x2, uint32_t& x3) {
  uint32_t t01 = add(x0, x1), t23 = add(x2, x3), t0123 = add(t01, t23);
  uint32_t t01123 = add(t0123, x1), t01233 = add(t0123, x3);
  uint32_t y3 = add(dbl(x0), t01233);
  uint32_t y1 = add(dbl(x2), t01123);
  x0 = add(t01, t01123);
  x2 = add(t23, t01233);
  x1 = y1;
  x3 = y3;
}

LG_HD void p2_external(uint32_t s[24]) {
#pragma unroll
  for (int c = 0; c < 6; c++) p2_m4(s[4 * c], s[4 * c + 1], s[4 * c + 2], s[4 * c + 3]);
  uint32_t t0 = s[0], t1 = s[1], t2 = s[2], t3 = s[3];
#pragma unroll
  for (int c = 1; c < 6; c++) {
    t0 = add(t0, s[4 * c]); t1 = add(t1, s[4 * c + 1]);
    t2 = add(t2, s[4 * c + 2]); t3 = add(t3, s[4 * c + 3]);
  }
#pragma unroll
  for (int c = 0; c < 6; c++) {
    s[4 * c] = add(s[4 * c], t0); s[4 * c + 1] = add(s[4 * c + 1], t1);
    s[4 * c + 2] = add(s[4 * c + 2], t2); s[4 * c + 3] = add(s[4 * c + 3], t3);
  }
}

LG_HD void p2_internal(uint32_t s[24]) {
  // pairwise sum: 5 dependent additions instead of 23
  uint32_t t[12];
#pragma unroll
  for (int i = 0; i < 12; i++) t[i] = add(s[2 * i], s[2 * i + 1]);
#pragma unroll
  for (int i = 0; i < 6; i++) t[i] = add(t[2 * i], t[2 * i + 1]);
#pragma unroll
  for (int i = 0; i < 3; i++) t[i] = add(t[2 * i], t[2 * i + 1]);
  const uint32_t sum = add(add(t[0], t[1]), t[2]);
#pragma unroll
  for (int i = 0; i < 24; i++) s[i] = add(sum, mul(s[i], LG_P2_DIAG[i]));
}

LG_HD uint32_t p2_cube(uint32_t x) { return mul(mul_lazy(x, x), x); }

// Unrolling of the round loops.  A fully unrolled permutation is ~9K
// instructions, more than the SM's instruction caches hold when warps drift
// apart; rolled round loops keep the hot code small.
#ifndef LG_P2_FULL_UNROLL
#define LG_P2_FULL_UNROLL 1
#endif
#ifndef LG_P2_PARTIAL_UNROLL
#define LG_P2_PARTIAL_UNROLL 3
#endif
#define LG_PRAGMA(x) _Pragma(#x)
#define LG_UNROLL(n) LG_PRAGMA(unroll n)

LG_HD void p2_full_round(uint32_t s[24], const uint32_t* rk) {
#pragma unroll
  for (int i = 0; i < 24; i++) s[i] = p2_cube(add(s[i], rk[i]));
  p2_external(s);
}

// Pairwise sum of v[0..N): depth log2(N) instead of N - 1.
template <int N> LG_HD uint32_t tree_sum(const uint32_t* v) {
  if constexpr (N == 1) return v[0];
  else return add(tree_sum<N / 2>(v), tree_sum<N - N / 2>(v + N / 2));
}

// Sum of N values in [0, p) as a 64-bit integer (two instructions a term,
// against three for a reduced addition), reduced once: with v < 2^37,
// v = hi 2^32 + lo = lo + hi (2^32 mod p); 2^32 mod p is MONT_ONE.
template <int N> LG_HD uint32_t wide_sum(const uint32_t* v) {
  static_assert(N <= 32, "the sum must stay below 2^37");
  uint64_t acc = 0;
#pragma unroll
  for (int i = 0; i < N; i++) acc += v[i];
  const uint64_t t = (uint64_t)(uint32_t)(acc >> 32) * MONT_ONE + (uint32_t)acc;  // < 2^32 + 2^30
  const uint32_t r = (uint32_t)t + (uint32_t)(t >> 32) * MONT_ONE;               // < 2^32
  return red(red(r));                                                            // [0, 2^32) -> [0, p)
}

constexpr uint32_t P2_DIAG_C[24] = LG_P2_DIAG_INIT;
static_assert(P2_DIAG_C[1] == MONT_ONE, "internal diagonal entry 1 is 1");

// The internal diagonal as canonical constants with their Shoup companions
// (products by d_i need no 64-bit multiply), and 23 for the carried sum.
struct P2DiagShoup { uint32_t w[24], ws[24]; };
constexpr P2DiagShoup make_p2_diag_shoup() {
  P2DiagShoup d{};
  for (int i = 0; i < 24; i++) {
    d.w[i] = cx_from_mont(P2_DIAG_C[i]);
    d.ws[i] = shoup(d.w[i]);
  }
  return d;
}
constexpr P2DiagShoup P2_DSH_H = make_p2_diag_shoup();
static_assert(P2_DSH_H.w[1] == 1, "internal diagonal entry 1 is 1");
static_assert(P2_DSH_H.w[0] == P - 2, "internal diagonal entry 0 is -2: s_0 <- sum + d_0 u = R - u");
#ifdef __CUDACC__
__constant__ P2DiagShoup P2_DSH_D = make_p2_diag_shoup();
#endif
#ifdef __CUDA_ARCH__
#define LG_P2_DSH P2_DSH_D
#else
#define LG_P2_DSH P2_DSH_H
#endif
constexpr uint32_t C23 = 23, C23_SH = shoup(23);

// Products by the diagonal entries +-2^-k (17 of the 24).  With
// x = hi 2^k + lo (lo < 2^k) and 2^k (p - 1)/2^k = p - 1 = -1 mod p,
//   x 2^-k = hi + lo 2^-k = hi - lo (p - 1)/2^k  (mod p):
// a shift, a mask and one multiply by a small constant in place of Shoup's
// three multiplies.  For x < 2p both hi and lo (p - 1)/2^k are below p, so
// t = +-(hi - lo c) lies in (-p, p) and min(t, t + p) on unsigned words is
// its residue in [0, p).  Montgomery words need no conversion (linear map).
template <int K, bool NEG> LG_HD uint32_t mul_pow2_inv(uint32_t x) {
  static_assert(K >= 1 && K <= 24, "p - 1 = 127 2^24");
  constexpr uint32_t c = (P - 1) >> K;
  const uint32_t lo = x & ((1u << K) - 1), hi = x >> K;
  const uint32_t t = NEG ? lo * c - hi : hi - lo * c;
  return umin(t, t + P);
}
constexpr uint32_t cx_pow2_inv(int k, bool neg) {
  const uint32_t v = cx_pow((P + 1) / 2, (uint64_t)k);
  return neg ? (P - v) % P : v;
}
#define LG_P2_DIAG_POW2(i, k, neg) \
  static_assert(P2_DSH_H.w[i] == cx_pow2_inv(k, neg), "internal diagonal entry " #i " is " #neg " 2^-" #k)
LG_P2_DIAG_POW2(3, 1, false);
LG_P2_DIAG_POW2(6, 1, true);
LG_P2_DIAG_POW2(9, 8, false);
LG_P2_DIAG_POW2(10, 2, false);
LG_P2_DIAG_POW2(11, 3, false);
LG_P2_DIAG_POW2(12, 4, false);
LG_P2_DIAG_POW2(13, 5, false);
LG_P2_DIAG_POW2(14, 6, false);
LG_P2_DIAG_POW2(15, 24, false);
LG_P2_DIAG_POW2(16, 8, true);
LG_P2_DIAG_POW2(17, 3, true);
LG_P2_DIAG_POW2(18, 4, true);
LG_P2_DIAG_POW2(19, 5, true);
LG_P2_DIAG_POW2(20, 6, true);
LG_P2_DIAG_POW2(21, 7, true);
LG_P2_DIAG_POW2(22, 9, true);
LG_P2_DIAG_POW2(23, 24, true);
#undef LG_P2_DIAG_POW2

// d_i s_i for i = 2..23 into p[2..23], for s_i < 2p; outputs in [0, p).
// Entries 2, 4, 5, 7, 8 (2, 3, 4, -3, -4) use Shoup's products.
LG_HD void p2_diag_products(const uint32_t s[24], uint32_t p[24]) {
  p[2] = mulc(s[2], LG_P2_DSH.w[2], LG_P2_DSH.ws[2]);
  p[3] = mul_pow2_inv<1, false>(s[3]);
  p[4] = mulc(s[4], LG_P2_DSH.w[4], LG_P2_DSH.ws[4]);
  p[5] = mulc(s[5], LG_P2_DSH.w[5], LG_P2_DSH.ws[5]);
  p[6] = mul_pow2_inv<1, true>(s[6]);
  p[7] = mulc(s[7], LG_P2_DSH.w[7], LG_P2_DSH.ws[7]);
  p[8] = mulc(s[8], LG_P2_DSH.w[8], LG_P2_DSH.ws[8]);
  p[9] = mul_pow2_inv<8, false>(s[9]);
  p[10] = mul_pow2_inv<2, false>(s[10]);
  p[11] = mul_pow2_inv<3, false>(s[11]);
  p[12] = mul_pow2_inv<4, false>(s[12]);
  p[13] = mul_pow2_inv<5, false>(s[13]);
  p[14] = mul_pow2_inv<6, false>(s[14]);
  p[15] = mul_pow2_inv<24, false>(s[15]);
  p[16] = mul_pow2_inv<8, true>(s[16]);
  p[17] = mul_pow2_inv<3, true>(s[17]);
  p[18] = mul_pow2_inv<4, true>(s[18]);
  p[19] = mul_pow2_inv<5, true>(s[19]);
  p[20] = mul_pow2_inv<6, true>(s[20]);
  p[21] = mul_pow2_inv<7, true>(s[21]);
  p[22] = mul_pow2_inv<9, true>(s[22]);
  p[23] = mul_pow2_inv<24, true>(s[23]);
}

// Partial rounds (S-box on lane 0, internal layer 1.1^T + diag).  With
// R = s_1 + ... + s_23 carried from round to round, one round is
//   u = S(s_0 + c),  sum = u + R,  s_0 <- sum + d_0 u,  s_i <- sum + d_i s_i,
//   R <- 23 sum + sum_{i>=1} d_i s_i   (s_i before the update),
// which is the same linear map; the products d_i s_i and their sum no longer
// wait for the S-box, so a round's dependent chain is the S-box and two
// additions.  s_1 .. s_23 stay unreduced in [0, 2p) between rounds (their
// only consumer is the next product d_i s_i, which accepts them), saving two
// of the three instructions of each of their additions.
LG_HD void p2_partial_rounds(uint32_t s[24]) {
  uint32_t R = tree_sum<23>(s + 1);
  LG_UNROLL(LG_P2_PARTIAL_UNROLL)
  for (int r = 0; r < 21; r++) {
    const uint32_t u = p2_cube(add(s[0], LG_P2_PARTIAL_RK[r]));
    uint32_t p[24];
    p[1] = red(s[1]);  // d_1 = 1
    p2_diag_products(s, p);
    const uint32_t D = wide_sum<23>(p + 1);
    const uint32_t sum = add(u, R);
    s[0] = sub(R, u);  // sum + d_0 u with d_0 = -2
#pragma unroll
    for (int i = 1; i < 24; i++) s[i] = sum + p[i];
    R = add(mulc(sum, C23, C23_SH), D);
  }
#pragma unroll
  for (int i = 1; i < 24; i++) s[i] = red(s[i]);
}

LG_HD void p2_permute(uint32_t s[24]) {
  p2_external(s);
  LG_UNROLL(LG_P2_FULL_UNROLL)
  for (int r = 0; r < 3; r++) p2_full_round(s, LG_P2_FULL_RK[r]);
  p2_partial_rounds(s);
  LG_UNROLL(LG_P2_FULL_UNROLL)
  for (int r = 3; r < 6; r++) p2_full_round(s, LG_P2_FULL_RK[r]);
}

// node = first 8 lanes of Perm([tag, 0 x7, left, right])
// (internal/hash/poseidon2.go:409-422); tag given in Montgomery form.
LG_HD void p2_compress(uint32_t tag_m, const uint32_t l[8], const uint32_t r[8], uint32_t out[8]) {
  uint32_t s[24];
  s[0] = tag_m;
#pragma unroll
  for (int i = 1; i < 8; i++) s[i] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) { s[8 + i] = l[i]; s[16 + i] = r[i]; }
  p2_permute(s);
#pragma unroll
  for (int i = 0; i < 8; i++) out[i] = s[i];
}

// The host's permutation for the transcript (p2_host.cpp): the same map as
// p2_permute, vectorised when the CPU has AVX2.
void p2_permute_host(uint32_t s[24]);
// The same with a given vector width (2: AVX-512, 1: AVX2, 0: scalar; the
// caller checks the CPU has it) and the width p2_permute_host uses.
void p2_permute_host_at(uint32_t s[24], int level);
int p2_host_simd_level();

// Host sponge: width 24, rate 16, overwrite mode, no padding
// (internal/hash/poseidon2.go:165-255).
struct HostSponge {
  uint32_t state[24];
  uint32_t block[16];
  int len = 0;
  bool wrote = false;
  HostSponge() { reset(); }
  void reset() {
    for (int i = 0; i < 24; i++) state[i] = 0;
    for (int i = 0; i < 16; i++) block[i] = 0;
    len = 0;
    wrote = false;
  }
  void write(uint32_t x_mont) {
    block[len++] = x_mont;
    if (len == 16) {
      for (int i = 0; i < 16; i++) state[i] = block[i];
      p2_permute_host(state);
      for (int i = 0; i < 16; i++) block[i] = 0;
      len = 0;
      wrote = true;
    }
  }
  void sum(uint32_t out[8]) {
    if (!wrote && len == 0) { for (int i = 0; i < 8; i++) out[i] = 0; return; }
    if (len > 0) {
      for (int i = 0; i < len; i++) state[i] = block[i];
      p2_permute_host(state);
      for (int i = 0; i < 16; i++) block[i] = 0;
      len = 0;
      wrote = true;
    }
    for (int i = 0; i < 8; i++) out[i] = state[i];
  }
};

}  // namespace lg
