// Host Poseidon2 (width 24) for the Fiat-Shamir transcript: the transcript is
// a chain of sponge absorptions the host computes between device phases
// (challenges, claimed-value binding, query positions), so its latency adds to
// every proof.  With AVX-512 (checked at run time) the 24-word state lives in
// a 16-lane and an 8-lane vector; with AVX2 only, in three 8-lane vectors: Montgomery products as even/odd 32x32->64 multiplies,
// the M4 blocks of the external layer as in-lane shuffles, the partial rounds
// in the carried-sum form of p2_partial_rounds (poseidon2.cuh) with one
// horizontal sum per round.  Same permutation, same words as p2_permute.
#include "poseidon2.cuh"

#if defined(__x86_64__)
#include <immintrin.h>

#include <cstdlib>
#define LG_AVX2 __attribute__((target("avx2")))

namespace lg {
namespace {

// The scalar S-box chain of the partial rounds, shortened for the host: the
// cube of a Montgomery word x (x^3 R after the reduction) as one 93-bit
// product reduced once by Montgomery's method with 2^64 (x^3 R^3 2^-64 =
// x^3 R for R = 2^32) instead of two reductions by 2^32; and the additions
// on the chain as the minimum of two independent sums.
constexpr uint64_t neg_inv64() {  // -p^-1 mod 2^64 (Newton's iteration)
  uint64_t v = 1;
  for (int i = 0; i < 7; i++) v *= 2 - (uint64_t)P * v;
  return 0 - v;
}
constexpr uint64_t P_INV_NEG64 = neg_inv64();
static_assert((uint64_t)P * P_INV_NEG64 == ~(uint64_t)0, "-p^-1 mod 2^64");
inline uint32_t cube_host(uint32_t x) {
  const uint64_t x2 = (uint64_t)x * x;                               // < 2^62
  const unsigned __int128 t = (unsigned __int128)x2 * x;            // < 2^93 < p 2^64
  const uint64_t m = (uint64_t)t * P_INV_NEG64;
  const uint32_t r = (uint32_t)((t + (unsigned __int128)m * P) >> 64);  // < 2p
  return umin(r, r - P);
}
// a + k and a - b for reduced words, each a minimum of two sums that do not
// wait for each other (k - p and b: prepared off the chain)
inline uint32_t add_pre(uint32_t a, uint32_t k, uint32_t k_minus_p) { return umin(a + k, a + k_minus_p); }
inline uint32_t sub_pre(uint32_t a_plus_p, uint32_t a, uint32_t b) { return umin(a - b, a_plus_p - b); }

LG_AVX2 inline __m256i vp() { return _mm256_set1_epi32((int)P); }

// a + b mod p for a, b in [0, p)
LG_AVX2 inline __m256i vadd(__m256i a, __m256i b) {
  const __m256i s = _mm256_add_epi32(a, b);
  return _mm256_min_epu32(s, _mm256_sub_epi32(s, vp()));
}
// x in [0, 2p) -> [0, p)
LG_AVX2 inline __m256i vred(__m256i x) { return _mm256_min_epu32(x, _mm256_sub_epi32(x, vp())); }

// Montgomery product, b in [0, p), a in [0, 2^32): as mul() in field.cuh.
LG_AVX2 inline __m256i vmul(__m256i a, __m256i b) {
  const __m256i p = vp(), pinv = _mm256_set1_epi32((int)P_INV_NEG);
  const __m256i te = _mm256_mul_epu32(a, b);
  const __m256i to = _mm256_mul_epu32(_mm256_srli_epi64(a, 32), _mm256_srli_epi64(b, 32));
  const __m256i me = _mm256_mul_epu32(te, pinv), mo = _mm256_mul_epu32(to, pinv);
  const __m256i ue = _mm256_add_epi64(te, _mm256_mul_epu32(me, p));
  const __m256i uo = _mm256_add_epi64(to, _mm256_mul_epu32(mo, p));
  return vred(_mm256_blend_epi32(_mm256_srli_epi64(ue, 32), uo, 0xAA));
}
// the same without the final reduction: [0, 2p), a valid first operand of vmul
LG_AVX2 inline __m256i vmul_lazy(__m256i a, __m256i b) {
  const __m256i p = vp(), pinv = _mm256_set1_epi32((int)P_INV_NEG);
  const __m256i te = _mm256_mul_epu32(a, b);
  const __m256i to = _mm256_mul_epu32(_mm256_srli_epi64(a, 32), _mm256_srli_epi64(b, 32));
  const __m256i me = _mm256_mul_epu32(te, pinv), mo = _mm256_mul_epu32(to, pinv);
  const __m256i ue = _mm256_add_epi64(te, _mm256_mul_epu32(me, p));
  const __m256i uo = _mm256_add_epi64(to, _mm256_mul_epu32(mo, p));
  return _mm256_blend_epi32(_mm256_srli_epi64(ue, 32), uo, 0xAA);
}

LG_AVX2 inline __m256i vcube(__m256i x) { return vmul(vmul_lazy(x, x), x); }
// x + k for a constant vector k, as the minimum of two sums that do not wait
// for each other
LG_AVX2 inline __m256i vadd_k(__m256i x, __m256i k) {
  return _mm256_min_epu32(_mm256_add_epi32(x, k), _mm256_add_epi32(x, _mm256_sub_epi32(k, vp())));
}

// M4 on the two 4-word blocks of v: y_i = x_i + 2 x_{i+1} + (x_0 + x_1 + x_2 + x_3),
// indices mod 4 -- the matrix of p2_m4's addition chain.
LG_AVX2 inline __m256i vm4(__m256i v) {
  const __m256i r = _mm256_shuffle_epi32(v, _MM_SHUFFLE(0, 3, 2, 1));
  const __m256i e = vadd(v, vadd(r, r));
  const __m256i s1 = vadd(v, _mm256_shuffle_epi32(v, _MM_SHUFFLE(2, 3, 0, 1)));
  const __m256i t = vadd(s1, _mm256_shuffle_epi32(s1, _MM_SHUFFLE(1, 0, 3, 2)));
  return vadd(e, t);
}

LG_AVX2 inline void vexternal(__m256i v[3]) {
  for (int k = 0; k < 3; k++) v[k] = vm4(v[k]);
  const __m256i s = vadd(vadd(v[0], v[1]), v[2]);  // column sums of blocks (0,2,4) | (1,3,5)
  const __m256i tot = vadd(s, _mm256_permute2x128_si256(s, s, 0x01));
  for (int k = 0; k < 3; k++) v[k] = vadd(v[k], tot);
}

// sum of the 8 lanes of x (each in [0, p))
LG_AVX2 inline uint32_t vhsum(__m256i x) {
  x = vadd(x, _mm256_permute2x128_si256(x, x, 0x01));
  x = vadd(x, _mm256_shuffle_epi32(x, _MM_SHUFFLE(1, 0, 3, 2)));
  x = vadd(x, _mm256_shuffle_epi32(x, _MM_SHUFFLE(2, 3, 0, 1)));
  return (uint32_t)_mm256_cvtsi256_si32(x);
}

LG_AVX2 inline void vfull_round(__m256i v[3], const uint32_t* rk) {
  for (int k = 0; k < 3; k++)
    v[k] = vcube(vadd_k(v[k], _mm256_loadu_si256(reinterpret_cast<const __m256i*>(rk + 8 * k))));
  vexternal(v);
}

constexpr uint32_t MONT_23 = 0x2dffffd2u;  // 23 * 2^32 mod p

LG_AVX2 void p2_permute_avx2(uint32_t s[24]) {
  __m256i v[3];
  for (int k = 0; k < 3; k++) v[k] = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(s + 8 * k));
  __m256i dg[3];
  for (int k = 0; k < 3; k++) dg[k] = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(P2_DIAG_H + 8 * k));
  const __m256i zero = _mm256_setzero_si256();
  vexternal(v);
  for (int r = 0; r < 3; r++) vfull_round(v, P2_FULL_RK_H[r]);
  // partial rounds, carried R = s_1 + ... + s_23 (as p2_partial_rounds)
  // s_0 stays a scalar through the rounds (lane 0 of v[0] is not read until
  // the end); with d_0 = -2 its update sum + d_0 u is R - u, no product
  uint32_t R = vhsum(vadd(_mm256_blend_epi32(v[0], zero, 0x01), vadd(v[1], v[2])));
  uint32_t s0 = (uint32_t)_mm256_cvtsi256_si32(v[0]);
  for (int r = 0; r < 21; r++) {
    const uint32_t k = P2_PARTIAL_RK_H[r];
    const uint32_t u = cube_host(add_pre(s0, k, k - P));
    const __m256i p0 = vmul(v[0], dg[0]), p1 = vmul(v[1], dg[1]), p2 = vmul(v[2], dg[2]);
    const uint32_t D = vhsum(vadd(_mm256_blend_epi32(p0, zero, 0x01), vadd(p1, p2)));
    const uint32_t sum = add(u, R);
    const __m256i sv = _mm256_set1_epi32((int)sum);
    s0 = sub_pre(R + P, R, u);
    v[0] = _mm256_add_epi32(sv, p0);  // unreduced in [0, 2p) until the next product
    v[1] = _mm256_add_epi32(sv, p1);
    v[2] = _mm256_add_epi32(sv, p2);
    R = add(mul(sum, MONT_23), D);
  }
  v[0] = _mm256_blend_epi32(v[0], _mm256_set1_epi32((int)s0), 0x01);
  for (int k = 0; k < 3; k++) v[k] = vred(v[k]);
  for (int r = 3; r < 6; r++) vfull_round(v, P2_FULL_RK_H[r]);
  for (int k = 0; k < 3; k++) _mm256_storeu_si256(reinterpret_cast<__m256i*>(s + 8 * k), v[k]);
}

// AVX-512: lanes 0..15 in one 16-lane vector (four M4 blocks), lanes 16..23
// in an 8-lane one (two blocks); the same steps as p2_permute_avx2.
#define LG_AVX512 __attribute__((target("avx512f,avx2")))

LG_AVX512 inline __m512i zp() { return _mm512_set1_epi32((int)P); }
LG_AVX512 inline __m512i zadd(__m512i a, __m512i b) {
  const __m512i s = _mm512_add_epi32(a, b);
  return _mm512_min_epu32(s, _mm512_sub_epi32(s, zp()));
}
LG_AVX512 inline __m512i zred(__m512i x) { return _mm512_min_epu32(x, _mm512_sub_epi32(x, zp())); }
LG_AVX512 inline __m512i zmul(__m512i a, __m512i b) {
  const __m512i p = zp(), pinv = _mm512_set1_epi32((int)P_INV_NEG);
  const __m512i te = _mm512_mul_epu32(a, b);
  const __m512i to = _mm512_mul_epu32(_mm512_srli_epi64(a, 32), _mm512_srli_epi64(b, 32));
  const __m512i me = _mm512_mul_epu32(te, pinv), mo = _mm512_mul_epu32(to, pinv);
  const __m512i ue = _mm512_add_epi64(te, _mm512_mul_epu32(me, p));
  const __m512i uo = _mm512_add_epi64(to, _mm512_mul_epu32(mo, p));
  return zred(_mm512_mask_blend_epi32((__mmask16)0xAAAA, _mm512_srli_epi64(ue, 32), uo));
}
LG_AVX512 inline __m512i zmul_lazy(__m512i a, __m512i b) {  // [0, 2p)
  const __m512i p = zp(), pinv = _mm512_set1_epi32((int)P_INV_NEG);
  const __m512i te = _mm512_mul_epu32(a, b);
  const __m512i to = _mm512_mul_epu32(_mm512_srli_epi64(a, 32), _mm512_srli_epi64(b, 32));
  const __m512i me = _mm512_mul_epu32(te, pinv), mo = _mm512_mul_epu32(to, pinv);
  const __m512i ue = _mm512_add_epi64(te, _mm512_mul_epu32(me, p));
  const __m512i uo = _mm512_add_epi64(to, _mm512_mul_epu32(mo, p));
  return _mm512_mask_blend_epi32((__mmask16)0xAAAA, _mm512_srli_epi64(ue, 32), uo);
}
LG_AVX512 inline __m512i zcube(__m512i x) { return zmul(zmul_lazy(x, x), x); }
LG_AVX512 inline __m512i zadd_k(__m512i x, __m512i k) {  // as vadd_k
  return _mm512_min_epu32(_mm512_add_epi32(x, k), _mm512_add_epi32(x, _mm512_sub_epi32(k, zp())));
}
LG_AVX512 inline __m512i zm4(__m512i v) {  // p2_m4 on each 128-bit lane, as vm4
  const __m512i r = _mm512_shuffle_epi32(v, (_MM_PERM_ENUM)_MM_SHUFFLE(0, 3, 2, 1));
  const __m512i e = zadd(v, zadd(r, r));
  const __m512i s1 = zadd(v, _mm512_shuffle_epi32(v, (_MM_PERM_ENUM)_MM_SHUFFLE(2, 3, 0, 1)));
  const __m512i t = zadd(s1, _mm512_shuffle_epi32(s1, (_MM_PERM_ENUM)_MM_SHUFFLE(1, 0, 3, 2)));
  return zadd(e, t);
}
LG_AVX512 inline void zexternal(__m512i& a, __m256i& b) {
  a = zm4(a);
  b = vm4(b);
  __m512i t = zadd(a, _mm512_shuffle_i32x4(a, a, _MM_SHUFFLE(1, 0, 3, 2)));  // blocks 0+2, 1+3
  t = zadd(t, _mm512_shuffle_i32x4(t, t, _MM_SHUFFLE(2, 3, 0, 1)));          // all four, in every lane
  const __m256i u = vadd(b, _mm256_permute2x128_si256(b, b, 0x01));         // blocks 4+5
  const __m512i tot = zadd(t, _mm512_broadcast_i32x4(_mm256_castsi256_si128(u)));
  a = zadd(a, tot);
  b = vadd(b, _mm512_castsi512_si256(tot));
}
LG_AVX512 inline void zfull_round(__m512i& a, __m256i& b, const uint32_t* rk) {
  a = zcube(zadd_k(a, _mm512_loadu_si512(rk)));
  b = vcube(vadd_k(b, _mm256_loadu_si256(reinterpret_cast<const __m256i*>(rk + 16))));
  zexternal(a, b);
}

// lanes 1..23 of (x, y) summed (each in [0, p))
LG_AVX512 inline uint32_t zsum_tail(__m512i x, __m256i y) {
  x = _mm512_mask_blend_epi32((__mmask16)0x0001, x, _mm512_setzero_si512());
  return vhsum(vadd(vadd(_mm512_castsi512_si256(x), _mm512_extracti64x4_epi64(x, 1)), y));
}

LG_AVX512 void p2_permute_avx512(uint32_t s[24]) {
  __m512i a = _mm512_loadu_si512(s);
  __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(s + 16));
  const __m512i da = _mm512_loadu_si512(P2_DIAG_H);
  const __m256i db = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(P2_DIAG_H + 16));
  zexternal(a, b);
  for (int r = 0; r < 3; r++) zfull_round(a, b, P2_FULL_RK_H[r]);
  // partial rounds, carried R = s_1 + ... + s_23 (as p2_partial_rounds)
  // s_0 as a scalar through the rounds, updated as R - u (d_0 = -2)
  uint32_t R = zsum_tail(a, b);
  uint32_t s0 = (uint32_t)_mm_cvtsi128_si32(_mm512_castsi512_si128(a));
  for (int r = 0; r < 21; r++) {
    const uint32_t k = P2_PARTIAL_RK_H[r];
    const uint32_t u = cube_host(add_pre(s0, k, k - P));
    const __m512i pa = zmul(a, da);
    const __m256i pb = vmul(b, db);
    const uint32_t D = zsum_tail(pa, pb);
    const uint32_t sum = add(u, R);
    const __m512i sv = _mm512_set1_epi32((int)sum);
    s0 = sub_pre(R + P, R, u);
    a = _mm512_add_epi32(sv, pa);  // unreduced in [0, 2p) until the next product
    b = _mm256_add_epi32(_mm512_castsi512_si256(sv), pb);
    R = add(mul(sum, MONT_23), D);
  }
  a = _mm512_mask_blend_epi32((__mmask16)0x0001, zred(a), _mm512_set1_epi32((int)s0));
  b = vred(b);
  for (int r = 3; r < 6; r++) zfull_round(a, b, P2_FULL_RK_H[r]);
  _mm512_storeu_si512(s, a);
  _mm256_storeu_si256(reinterpret_cast<__m256i*>(s + 16), b);
}

// 2: AVX-512, 1: AVX2, 0: neither
int cpu_simd_level() {
  __builtin_cpu_init();
  if (__builtin_cpu_supports("avx512f") && !getenv("LOOM_B200_NO_AVX512")) return 2;
  return __builtin_cpu_supports("avx2") ? 1 : 0;
}

}  // namespace

void p2_permute_host_at(uint32_t s[24], int level) {
  if (level >= 2)
    p2_permute_avx512(s);
  else if (level == 1)
    p2_permute_avx2(s);
  else
    p2_permute(s);
}
int p2_host_simd_level() {
  static const int simd = cpu_simd_level();
  return simd;
}
void p2_permute_host(uint32_t s[24]) { p2_permute_host_at(s, p2_host_simd_level()); }

}  // namespace lg

#else
namespace lg {
void p2_permute_host_at(uint32_t s[24], int) { p2_permute(s); }
int p2_host_simd_level() { return 0; }
void p2_permute_host(uint32_t s[24]) { p2_permute(s); }
}  // namespace lg
#endif
