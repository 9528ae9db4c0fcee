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
  uint32_t sum = s[0];
#pragma unroll
  for (int i = 1; i < 24; i++) sum = add(sum, s[i]);
#pragma unroll
  for (int i = 0; i < 24; i++) s[i] = add(sum, mul(s[i], LG_P2_DIAG[i]));
}

LG_HD uint32_t p2_cube(uint32_t x) { return mul(sqr(x), x); }

LG_HD void p2_permute(uint32_t s[24]) {
  p2_external(s);
#pragma unroll
  for (int r = 0; r < 3; r++) {
#pragma unroll
    for (int i = 0; i < 24; i++) s[i] = p2_cube(add(s[i], LG_P2_FULL_RK[r][i]));
    p2_external(s);
  }
#pragma unroll 3
  for (int r = 0; r < 21; r++) {
    s[0] = p2_cube(add(s[0], LG_P2_PARTIAL_RK[r]));
    p2_internal(s);
  }
#pragma unroll
  for (int r = 3; r < 6; r++) {
#pragma unroll
    for (int i = 0; i < 24; i++) s[i] = p2_cube(add(s[i], LG_P2_FULL_RK[r][i]));
    p2_external(s);
  }
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
      p2_permute(state);
      for (int i = 0; i < 16; i++) block[i] = 0;
      len = 0;
      wrote = true;
    }
  }
  void sum(uint32_t out[8]) {
    if (!wrote && len == 0) { for (int i = 0; i < 8; i++) out[i] = 0; return; }
    if (len > 0) {
      for (int i = 0; i < len; i++) state[i] = block[i];
      p2_permute(state);
      for (int i = 0; i < 16; i++) block[i] = 0;
      len = 0;
      wrote = true;
    }
    for (int i = 0; i < 8; i++) out[i] = state[i];
  }
};

}  // namespace lg
