// Cooperative Poseidon2 width 24: six lanes of a warp share one permutation.
// Lane i of a group (i = lane % 6, groups of lanes 0-5, 6-11, ..., 24-29)
// holds state[4i .. 4i+3], one chunk of the external layer's M4 blocks, so
// circ(2 M4, M4, ...) is lane-local except for its four column sums, and the
// internal layer needs one sum over the group.  Both are 3-shuffle
// all-reductions over the six lanes.  Lanes 30 and 31 run the same code on
// dummy data so every shuffle has the full warp.
//
// Per permutation this issues about the same instructions as one thread
// running it alone, but the dependent chain is six times shorter: the Merkle
// tree tops and the injection chains, which have little parallelism, are
// latency bound.  Round structure as recursion/p2_air.go:206-300.
#pragma once
#include "poseidon2.cuh"

namespace lg {

struct P2Lane {
  int lane, base, idx;    // warp lane, first lane of the group, index in the group (0..5)
  uint32_t dw[4], dws[4];  // internal diagonal (canonical, Shoup companion) of this lane's four elements
  __device__ __forceinline__ void init() {
    lane = threadIdx.x & 31;
    idx = lane % 6;
    base = lane - idx;
    for (int i = 0; i < 4; i++) {
      dw[i] = P2_DSH_D.w[(4 * idx + i) % 24];
      dws[i] = P2_DSH_D.ws[(4 * idx + i) % 24];
    }
  }
  __device__ __forceinline__ int at(int k) const { return (base + ((idx + k) % 6)) & 31; }
  // sum over the group's six lanes, in every lane
  __device__ __forceinline__ uint32_t allreduce(uint32_t v) const {
    uint32_t s1 = add(v, __shfl_sync(0xffffffffu, v, (base + (idx ^ 1)) & 31));
    uint32_t s2 = add(s1, __shfl_sync(0xffffffffu, s1, at(2)));
    return add(s2, __shfl_sync(0xffffffffu, s1, at(4)));
  }
};

// Full-round keys staged in shared memory (lane-dependent indices).
__device__ __forceinline__ void p2_load_full_keys(uint32_t* smem_keys /*144 words*/) {
  for (int i = threadIdx.x; i < 144; i += blockDim.x) smem_keys[i] = (&P2_FULL_RK_D[0][0])[i];
  __syncthreads();
}

__device__ __forceinline__ void p2c_external(uint32_t x[4], const P2Lane& L) {
  p2_m4(x[0], x[1], x[2], x[3]);
  uint32_t c0 = L.allreduce(x[0]), c1 = L.allreduce(x[1]), c2 = L.allreduce(x[2]), c3 = L.allreduce(x[3]);
  x[0] = add(x[0], c0);
  x[1] = add(x[1], c1);
  x[2] = add(x[2], c2);
  x[3] = add(x[3], c3);
}

__device__ __forceinline__ void p2c_full(uint32_t x[4], const P2Lane& L, const uint32_t* keys /*24 words*/) {
#pragma unroll
  for (int i = 0; i < 4; i++) x[i] = p2_cube(add(x[i], keys[(4 * L.idx + i) % 24]));
  p2c_external(x, L);
}

__device__ __forceinline__ void p2c_permute(uint32_t x[4], const P2Lane& L, const uint32_t* smem_keys) {
  p2c_external(x, L);
#pragma unroll
  for (int r = 0; r < 3; r++) p2c_full(x, L, smem_keys + 24 * r);
  // Partial rounds as p2_partial_rounds: R = s_1 + ... + s_23 is carried,
  // and every lane of the group carries its own copy of s_0 (the same
  // values in all six), so the S-box output needs no broadcast: a round's
  // dependent chain is the S-box and two additions, while the group sum of
  // d_i s_i for the next R runs beside it.
  uint32_t s0 = __shfl_sync(0xffffffffu, x[0], L.base & 31);
  uint32_t R = L.allreduce(add(add(L.idx ? x[0] : 0u, x[1]), add(x[2], x[3])));
#pragma unroll 3
  for (int r = 0; r < 21; r++) {
    uint32_t p[4];
#pragma unroll
    for (int i = 0; i < 4; i++) p[i] = mulc(x[i], L.dw[i], L.dws[i]);
    const uint32_t D = L.allreduce(add(add(L.idx ? p[0] : 0u, p[1]), add(p[2], p[3])));
    const uint32_t u = p2_cube(add(s0, P2_PARTIAL_RK_D[r]));
    const uint32_t sum = add(u, R);
    s0 = sub(R, u);  // sum + d_0 u with d_0 = -2
    x[0] = L.idx ? add(sum, p[0]) : s0;
#pragma unroll
    for (int i = 1; i < 4; i++) x[i] = sum + p[i];  // unreduced in [0, 2p) until the next product
    R = add(mulc(sum, C23, C23_SH), D);
  }
#pragma unroll
  for (int i = 1; i < 4; i++) x[i] = red(x[i]);
#pragma unroll
  for (int r = 3; r < 6; r++) p2c_full(x, L, smem_keys + 24 * r);
}

// Node compression H(left, right) with the digests held as: left in lanes
// idx 2, 3 and right in lanes idx 4, 5 (4 words each); the result lands in
// lanes idx 0, 1.
__device__ __forceinline__ void p2c_compress(uint32_t x[4], const P2Lane& L, const uint32_t* smem_keys) {
  if (L.idx == 0) { x[0] = to_mont(0x4e4f4445u); x[1] = x[2] = x[3] = 0; }
  if (L.idx == 1) { x[0] = x[1] = x[2] = x[3] = 0; }
  p2c_permute(x, L, smem_keys);
}

// Moves a digest from lanes idx 0, 1 to lanes idx 2, 3 (the left input slot).
__device__ __forceinline__ void p2c_digest_to_left(uint32_t x[4], const P2Lane& L) {
  uint32_t y[4];
#pragma unroll
  for (int i = 0; i < 4; i++) y[i] = __shfl_sync(0xffffffffu, x[i], (L.base + ((L.idx + 4) % 6)) & 31);
  if (L.idx == 2 || L.idx == 3)
#pragma unroll
    for (int i = 0; i < 4; i++) x[i] = y[i];
}

}  // namespace lg
