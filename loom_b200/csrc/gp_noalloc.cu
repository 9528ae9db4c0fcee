// Grand product without any device allocation: lg_grand_product_noalloc.
//
// Who needs it: callers that cannot call cudaMalloc — code running where a
// caching allocator owns the device memory and forbids raw allocations, code
// inside a memory-capped sandbox, or a host that must not add allocation
// latency to its request path.  They pass inputs and outputs they already
// own; the only scratch this entry point uses is the file-scope device array
// below (the tile totals and their prefix products), which every GPU that
// loads this library holds until the process exits.
//
// Same result as lg_grand_product: out[0] = 1, out[i] = prod_{k<i} num[k]/den[k].
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/loom_gpu.h"
#include "field.cuh"

namespace lg {
// Kernel launch counter of the library (lg_kernel_launches), defined with the
// other entry points.
void note_launches(uint64_t k);
}  // namespace lg

namespace {

using namespace lg;

constexpr uint64_t NOALLOC_GP_MAX_ROWS = 1ull << 22;  // the largest loom module (2^22 rows)
constexpr int NA_THREADS = 256, NA_PER_THREAD = 8, NA_TILE = NA_THREADS * NA_PER_THREAD;
constexpr uint32_t NA_MAX_TILES = (uint32_t)(NOALLOC_GP_MAX_ROWS / NA_TILE);  // 2048

// Tile totals [0, 6 * NA_MAX_TILES) and their exclusive prefix products
// [6 * NA_MAX_TILES, 12 * NA_MAX_TILES): 96 KiB.  Every word a call reads is
// written earlier in the same call, so nothing has to be cleared.
static __device__ __align__(256) uint32_t g_gp_scratch[12 * NA_MAX_TILES];

__device__ __forceinline__ E6 ld_row(const uint32_t* p, uint64_t i) {
  E6 r;
  for (int w = 0; w < 6; w++) r.c[w] = p[6 * i + w];
  return r;
}
__device__ __forceinline__ void st_row(uint32_t* p, uint64_t i, const E6& v) {
  for (int w = 0; w < 6; w++) p[6 * i + w] = v.c[w];
}

__global__ void k_na_ratio(const uint32_t* num, const uint32_t* den, uint64_t n, uint32_t* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  st_row(out, i, e6_mul(ld_row(num, i), e6_inv(ld_row(den, i))));
}

// In-place exclusive product scan inside each tile of NA_TILE rows; the tile
// product goes to totals[6 t + w].
__global__ void k_na_scan(uint32_t* x, uint64_t n, uint32_t* totals) {
  __shared__ E6 part[NA_THREADS];
  const uint64_t base = (uint64_t)blockIdx.x * NA_TILE + (uint64_t)threadIdx.x * NA_PER_THREAD;
  E6 v[NA_PER_THREAD];
  E6 acc = e6_one();
  for (int i = 0; i < NA_PER_THREAD; i++) {
    v[i] = acc;  // product of this thread's rows before row i
    uint64_t idx = base + i;
    if (idx < n) acc = e6_mul(acc, ld_row(x, idx));
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int off = 1; off < NA_THREADS; off <<= 1) {
    E6 t = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : e6_one();
    __syncthreads();
    if (threadIdx.x >= (unsigned)off) part[threadIdx.x] = e6_mul(part[threadIdx.x], t);
    __syncthreads();
  }
  const E6 pre = threadIdx.x ? part[threadIdx.x - 1] : e6_one();
  for (int i = 0; i < NA_PER_THREAD; i++) {
    uint64_t idx = base + i;
    if (idx < n) st_row(x, idx, e6_mul(pre, v[i]));
  }
  if (threadIdx.x == NA_THREADS - 1)
    for (int w = 0; w < 6; w++) totals[6 * blockIdx.x + w] = part[NA_THREADS - 1].c[w];
}

__global__ void k_na_prefix(const uint32_t* totals, uint32_t nt, uint32_t* pre) {
  E6 acc = e6_one();
  for (uint32_t t = 0; t < nt; t++) {
    for (int w = 0; w < 6; w++) pre[6 * t + w] = acc.c[w];
    E6 v;
    for (int w = 0; w < 6; w++) v.c[w] = totals[6 * t + w];
    acc = e6_mul(acc, v);
  }
}

__global__ void k_na_apply(uint32_t* x, uint64_t n, const uint32_t* pre) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t t = i / NA_TILE;
  E6 p;
  for (int w = 0; w < 6; w++) p.c[w] = pre[6 * t + w];
  st_row(x, i, e6_mul(p, ld_row(x, i)));
}

// Device address of g_gp_scratch, looked up once per device with that
// device current (host code cannot use the symbol's name as a pointer).
std::mutex g_mu;
constexpr int MAX_DEVICES = 64;
uint32_t* g_scratch_ptr[MAX_DEVICES] = {};

int scratch_for_current_device(uint32_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LG_ERR_CUDA;
  if (dev < 0 || dev >= MAX_DEVICES) return LG_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_gp_scratch) != cudaSuccess || !p) return LG_ERR_CUDA;
    g_scratch_ptr[dev] = (uint32_t*)p;
  }
  *out = g_scratch_ptr[dev];
  return LG_OK;
}

}  // namespace

extern "C" int lg_grand_product_noalloc(const uint32_t* num, const uint32_t* den, uint64_t n, uint32_t* out,
                                        void* stream) {
  if (!num || !den || !out || n == 0) return LG_ERR_INVALID;
  if (n > NOALLOC_GP_MAX_ROWS) return LG_ERR_UNSUPPORTED;
  // An error already pending on this thread (from the caller's own work) is
  // left in place and reported, not cleared and taken for one of ours.
  if (cudaPeekAtLastError() != cudaSuccess) return LG_ERR_CUDA;
  uint32_t* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != LG_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t nt = (uint32_t)((n + NA_TILE - 1) / NA_TILE);
  uint32_t* totals = scratch;
  uint32_t* pre = scratch + 6 * NA_MAX_TILES;
  const unsigned g = (unsigned)((n + 255) / 256);
  k_na_ratio<<<g, 256, 0, st>>>(num, den, n, out);
  k_na_scan<<<nt, NA_THREADS, 0, st>>>(out, n, totals);
  k_na_prefix<<<1, 1, 0, st>>>(totals, nt, pre);
  k_na_apply<<<g, 256, 0, st>>>(out, n, pre);
  note_launches(4);
  return cudaGetLastError() == cudaSuccess ? LG_OK : LG_ERR_CUDA;
}
