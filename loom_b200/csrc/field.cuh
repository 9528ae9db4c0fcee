// KoalaBear field (p = 2^31 - 2^24 + 1) in Montgomery form, R = 2^32: the
// word layout of gnark-crypto's koalabear.Element, so buffers coming from
// the Go prover (trace columns, []ext.E6) are used as they are.
//
// E6 = E2[v]/(v^3 - (u + 1)), E2 = F[u]/(u^2 - 3) (recursion/e6.go:21-53),
// coefficient order [B0.A0, B0.A1, B1.A0, B1.A1, B2.A0, B2.A1]
// (internal/hash/hash.go:59-68).  Products use Karatsuba at both levels
// (3 base products per E2 product, 6 E2 products per E6 product).
//
// Every function is __host__ __device__: the host-side Fiat-Shamir transcript
// uses the same code as the kernels.
#pragma once
#ifdef __CUDACC_RTC__  // compiled at run time (the constraint kernels, xjit.cuh): no host headers
typedef unsigned char uint8_t;
typedef unsigned int uint32_t;
typedef int int32_t;
typedef unsigned long long uint64_t;
typedef long long int64_t;
#else
#include <cstdint>
#endif

#ifdef __CUDACC__
#define LG_HD __host__ __device__ __forceinline__
#else
#define LG_HD inline
#endif

namespace lg {

constexpr uint32_t P = 0x7f000001u;
constexpr uint32_t P_INV_NEG = 0x7effffffu;  // -p^-1 mod 2^32
constexpr uint32_t MONT_ONE = 0x01fffffeu;   // 2^32 mod p
constexpr uint32_t R2 = 0x17f7efe4u;         // 2^64 mod p (to_mont helper)

// Reductions use min(x, x - p) on unsigned words: when x < p the
// subtraction wraps above x, so the minimum is the reduced value without a
// branch or predicate.
LG_HD uint32_t umin(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return ::min(a, b);
#else
  return a < b ? a : b;
#endif
}
LG_HD uint32_t add(uint32_t a, uint32_t b) { uint32_t s = a + b; return umin(s, s - P); }
LG_HD uint32_t sub(uint32_t a, uint32_t b) { uint32_t d = a - b; return umin(d, d + P); }
LG_HD uint32_t neg(uint32_t a) { return a ? P - a : 0; }
// a - b + p, in (0, 2p) for a, b < p: unreduced, for the first operand of mul
LG_HD uint32_t sub_lazy(uint32_t a, uint32_t b) { return a + (P - b); }
// x in [0, 2p) -> [0, p)
LG_HD uint32_t red(uint32_t x) { return umin(x, x - P); }
LG_HD uint32_t dbl(uint32_t a) { return add(a, a); }

// Montgomery product a*b*2^-32 mod p, output in [0, p).  Inputs: b in
// [0, p) and a in [0, p) or, unreduced, anywhere in [0, 2^32): then
// t + m p < 2^33 p < 2^64 and the quotient stays below 2p.
LG_HD uint32_t mul(uint32_t a, uint32_t b) {
  uint64_t t = (uint64_t)a * b;
  uint32_t m = (uint32_t)t * P_INV_NEG;
  uint64_t u = t + (uint64_t)m * P;
  uint32_t r = (uint32_t)(u >> 32);
  return umin(r, r - P);
}
LG_HD uint32_t sqr(uint32_t a) { return mul(a, a); }

// Product by a fixed constant w (canonical, < p) with its precomputed
// companion ws = floor(w 2^32 / p) (Shoup's precomputed-quotient method):
// q = hi(x ws) under-estimates floor(x w / p) by at most one, so
// r = x w - q p (mod 2^32) lies in [0, 2p) for every x < 2^32, unreduced
// inputs included.  Three 32-bit multiplies, no 64-bit product.  Montgomery
// words need no conversion: (x R) w = (x w) R.
constexpr uint32_t shoup(uint32_t w) { return (uint32_t)(((uint64_t)w << 32) / P); }
LG_HD uint32_t umulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}
LG_HD uint32_t mulc_lazy(uint32_t x, uint32_t w, uint32_t ws) { return x * w - umulhi32(x, ws) * P; }
LG_HD uint32_t mulc(uint32_t x, uint32_t w, uint32_t ws) {
  const uint32_t r = mulc_lazy(x, w, ws);
  return umin(r, r - P);
}

// Compile-time field arithmetic on canonical values (constant tables).
constexpr uint32_t cx_mulmod(uint32_t a, uint32_t b) { return (uint32_t)((uint64_t)a * b % P); }
constexpr uint32_t cx_pow(uint32_t a, uint64_t e) {
  uint32_t r = 1;
  while (e) {
    if (e & 1) r = cx_mulmod(r, a);
    a = cx_mulmod(a, a);
    e >>= 1;
  }
  return r;
}
constexpr uint32_t cx_from_mont(uint32_t m) { return cx_mulmod(m, cx_pow(MONT_ONE, P - 2)); }
// Montgomery product without the final reduction: result in [0, 2p) for
// inputs in [0, p); fit to feed mul() as its unreduced operand.
LG_HD uint32_t mul_lazy(uint32_t a, uint32_t b) {
  uint64_t t = (uint64_t)a * b;
  uint32_t m = (uint32_t)t * P_INV_NEG;
  return (uint32_t)((t + (uint64_t)m * P) >> 32);
}
LG_HD uint32_t to_mont(uint32_t canonical) { return mul(canonical % P, R2); }
LG_HD uint32_t from_mont(uint32_t m) { return mul(m, 1u); }
LG_HD uint32_t mont_pow(uint32_t a, uint64_t e) {
  uint32_t r = MONT_ONE;
  while (e) { if (e & 1) r = mul(r, a); a = mul(a, a); e >>= 1; }
  return r;
}
LG_HD uint32_t inv(uint32_t a) { return mont_pow(a, P - 2); }

struct E2 { uint32_t a0, a1; };
struct E6 { uint32_t c[6]; };

LG_HD E2 e2_add(E2 x, E2 y) { return {add(x.a0, y.a0), add(x.a1, y.a1)}; }
LG_HD E2 e2_sub(E2 x, E2 y) { return {sub(x.a0, y.a0), sub(x.a1, y.a1)}; }
LG_HD uint32_t triple(uint32_t a) { return add(add(a, a), a); }
LG_HD E2 e2_mul(E2 x, E2 y) {
  uint32_t v0 = mul(x.a0, y.a0), v1 = mul(x.a1, y.a1);
  uint32_t m = mul(x.a0 + x.a1, add(y.a0, y.a1));  // first operand unreduced: < 2p
  return {add(v0, triple(v1)), sub(sub(m, v0), v1)};
}
// (p + q u)(1 + u) = (p + 3q) + (p + q) u
LG_HD E2 e2_mul_xi(E2 x) { return {add(x.a0, triple(x.a1)), add(x.a0, x.a1)}; }
LG_HD E2 e2_inv(E2 x) {
  uint32_t n = sub(sqr(x.a0), triple(sqr(x.a1)));
  uint32_t ni = inv(n);
  return {mul(x.a0, ni), mul(neg(x.a1), ni)};
}

LG_HD E2 g2(const E6& a, int i) { return {a.c[2 * i], a.c[2 * i + 1]}; }
LG_HD void s2(E6& a, int i, E2 v) { a.c[2 * i] = v.a0; a.c[2 * i + 1] = v.a1; }

LG_HD E6 e6_zero() { E6 r; for (int i = 0; i < 6; i++) r.c[i] = 0; return r; }
LG_HD E6 e6_one() { E6 r = e6_zero(); r.c[0] = MONT_ONE; return r; }
LG_HD E6 e6_base(uint32_t a) { E6 r = e6_zero(); r.c[0] = a; return r; }
LG_HD E6 e6_add(const E6& a, const E6& b) { E6 r; for (int i = 0; i < 6; i++) r.c[i] = add(a.c[i], b.c[i]); return r; }
LG_HD E6 e6_sub(const E6& a, const E6& b) { E6 r; for (int i = 0; i < 6; i++) r.c[i] = sub(a.c[i], b.c[i]); return r; }
LG_HD E6 e6_mul_base(const E6& a, uint32_t b) { E6 r; for (int i = 0; i < 6; i++) r.c[i] = mul(a.c[i], b); return r; }
LG_HD bool e6_eq(const E6& a, const E6& b) {
  for (int i = 0; i < 6; i++) if (a.c[i] != b.c[i]) return false;
  return true;
}

LG_HD E6 e6_mul(const E6& x, const E6& y) {
  E2 a0 = g2(x, 0), a1 = g2(x, 1), a2 = g2(x, 2);
  E2 b0 = g2(y, 0), b1 = g2(y, 1), b2 = g2(y, 2);
  E2 v0 = e2_mul(a0, b0), v1 = e2_mul(a1, b1), v2 = e2_mul(a2, b2);
  E2 t12 = e2_sub(e2_sub(e2_mul(e2_add(a1, a2), e2_add(b1, b2)), v1), v2);
  E2 t01 = e2_sub(e2_sub(e2_mul(e2_add(a0, a1), e2_add(b0, b1)), v0), v1);
  E2 t02 = e2_sub(e2_sub(e2_mul(e2_add(a0, a2), e2_add(b0, b2)), v0), v2);
  E6 r;
  s2(r, 0, e2_add(v0, e2_mul_xi(t12)));
  s2(r, 1, e2_add(t01, e2_mul_xi(v2)));
  s2(r, 2, e2_add(t02, v1));
  return r;
}
LG_HD E6 e6_sqr(const E6& x) { return e6_mul(x, x); }

// (c0, c1, c2) / (a0 c0 + xi (a2 c1 + a1 c2)) with c0 = a0^2 - xi a1 a2,
// c1 = xi a2^2 - a0 a1, c2 = a1^2 - a0 a2.
LG_HD E6 e6_inv(const E6& a) {
  E2 a0 = g2(a, 0), a1 = g2(a, 1), a2 = g2(a, 2);
  E2 c0 = e2_sub(e2_mul(a0, a0), e2_mul_xi(e2_mul(a1, a2)));
  E2 c1 = e2_sub(e2_mul_xi(e2_mul(a2, a2)), e2_mul(a0, a1));
  E2 c2 = e2_sub(e2_mul(a1, a1), e2_mul(a0, a2));
  E2 t = e2_add(e2_mul(a0, c0), e2_mul_xi(e2_add(e2_mul(a2, c1), e2_mul(a1, c2))));
  E2 ti = e2_inv(t);
  E6 r;
  s2(r, 0, e2_mul(c0, ti));
  s2(r, 1, e2_mul(c1, ti));
  s2(r, 2, e2_mul(c2, ti));
  return r;
}
LG_HD E6 e6_pow(E6 a, uint64_t e) {
  E6 r = e6_one();
  while (e) { if (e & 1) r = e6_mul(r, a); a = e6_mul(a, a); e >>= 1; }
  return r;
}

// Generator of the subgroup of order 2^logn: (3^127)^(2^(24-logn)), Montgomery.
LG_HD uint32_t root_of_unity_mont(int logn) {
  uint32_t w = mont_pow(to_mont(3), (P - 1) >> 24);
  for (int i = logn; i < 24; i++) w = mul(w, w);
  return w;
}

LG_HD uint32_t bitrev32(uint32_t x, int logn) {
#ifdef __CUDA_ARCH__
  return logn ? __brev(x) >> (32 - logn) : 0;
#else
  uint32_t r = 0;
  for (int i = 0; i < logn; i++) { r = (r << 1) | (x & 1); x >>= 1; }
  return r;
#endif
}

}  // namespace lg
