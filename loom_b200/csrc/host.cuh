// Host-side pieces of the prover: device memory, program descriptor,
// Fiat-Shamir transcript (internal/fiat-shamir/transcript.go:124-355) and the
// canonical proof writer.  Errors are C++ exceptions inside the library and
// become status codes at the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/loom_gpu.h"
#include "kernels.cuh"

namespace lg {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define LG_CK(x)                                                                                      \
  do {                                                                                                \
    cudaError_t e_ = (x);                                                                             \
    if (e_ != cudaSuccess)                                                                            \
      throw ::lg::Error(e_ == cudaErrorMemoryAllocation ? LG_ERR_OOM : LG_ERR_CUDA,     \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                             \
  } while (0)
// Every kernel launch is followed by LG_LAUNCH(): it checks the launch and
// counts it (lg_kernel_launches).
inline std::atomic<uint64_t> g_launches{0};
#define LG_LAUNCH()                                                                                 \
  do {                                                                                              \
    const cudaError_t e_ = cudaGetLastError();                                                      \
    if (e_ != cudaSuccess)                                                                          \
      throw ::lg::Error(LG_ERR_CUDA, std::string("kernel launch at ") + __FILE__ + ":" +              \
                                         std::to_string(__LINE__) + ": " + cudaGetErrorString(e_)); \
    ::lg::g_launches.fetch_add(1);                                                                  \
  } while (0)

// Device bytes held by one context (its DBuf allocations and arena chunks),
// their high-water mark, and an optional cap (lg_ctx_create's hbm_budget:
// an allocation past it fails with LG_ERR_OOM).  Calls on a context charge
// their allocations to it through g_mem_acct.
struct MemAcct {
  std::atomic<int64_t> held{0}, peak{0};
  int64_t budget = 0;  // bytes; 0 = no cap
  void charge(int64_t b) {
    const int64_t now = held.fetch_add(b) + b;
    if (budget && now > budget) {
      held.fetch_sub(b);
      throw Error(LG_ERR_OOM, "context HBM budget of " + std::to_string(budget) + " bytes exceeded (" +
                                  std::to_string(now) + " bytes needed)");
    }
    int64_t p = peak.load();
    while (now > p && !peak.compare_exchange_weak(p, now)) {}
  }
  void refund(int64_t b) { held.fetch_sub(b); }
};
inline thread_local MemAcct* g_mem_acct = nullptr;
struct AcctScope {
  MemAcct* prev;
  explicit AcctScope(MemAcct* a) : prev(g_mem_acct) { g_mem_acct = a; }
  ~AcctScope() { g_mem_acct = prev; }
  AcctScope(const AcctScope&) = delete;
  AcctScope& operator=(const AcctScope&) = delete;
};

// Prove-scoped device memory: the small buffers of one prove (upload tables,
// per-group scratch; about a thousand per prove) come from a bump arena of
// retained chunks instead of one stream-ordered pool allocation and free
// each.  The arena is rewound when the next call on the context starts, after
// its stream is idle; chunks are used on that context's stream only.
struct DevArena {
  static constexpr size_t MAX_OBJ = (size_t)1 << 20, CHUNK = (size_t)32 << 20, ALIGN = 256;
  std::vector<std::pair<uint8_t*, size_t>> chunks;
  size_t cur = 0, off = 0;
  MemAcct* acct = nullptr;  // charged for the chunks
  void* take(size_t bytes, cudaStream_t s) {
    bytes = (bytes + ALIGN - 1) & ~(ALIGN - 1);
    while (cur < chunks.size() && off + bytes > chunks[cur].second) {
      cur++;
      off = 0;
    }
    if (cur == chunks.size()) {
      uint8_t* p = nullptr;
      size_t sz = std::max(CHUNK, bytes);
      if (g_mem_acct) {
        if (acct && acct != g_mem_acct) throw Error(LG_ERR_INVALID, "device arena shared between contexts");
        g_mem_acct->charge((int64_t)sz);
        acct = g_mem_acct;
      }
      if (cudaMallocAsync((void**)&p, sz, s) != cudaSuccess) {
        cudaGetLastError();
        if (g_mem_acct) g_mem_acct->refund((int64_t)sz);
        throw Error(LG_ERR_OOM, "device arena chunk allocation failed");
      }
      chunks.push_back({p, sz});
      off = 0;
    }
    void* r = chunks[cur].first + off;
    off += bytes;
    return r;
  }
  void rewind() { cur = 0; off = 0; }
  void release(cudaStream_t s) {
    for (auto& c : chunks) {
      cudaFreeAsync(c.first, s);
      if (acct) acct->refund((int64_t)c.second);
    }
    chunks.clear();
    rewind();
  }
};
// The arena that this thread's small DBufs come from (null: pool allocations).
inline thread_local DevArena* g_dev_arena = nullptr;
struct ArenaScope {
  DevArena* prev;
  explicit ArenaScope(DevArena* a) : prev(g_dev_arena) { g_dev_arena = a; }
  ~ArenaScope() { g_dev_arena = prev; }
  ArenaScope(const ArenaScope&) = delete;
  ArenaScope& operator=(const ArenaScope&) = delete;
};

// Device buffer of u32 words, stream-ordered allocation (or a slice of the
// current prove's arena).
struct DBuf {
  uint32_t* p = nullptr;
  size_t words = 0;
  cudaStream_t st = nullptr;
  bool borrowed = false;  // caller-owned memory: never freed here
  MemAcct* acct = nullptr;  // charged for this allocation
  DBuf() = default;
  DBuf(size_t w, cudaStream_t s) : words(w), st(s) {
    if (!w) return;
    if (g_dev_arena && w * 4 <= DevArena::MAX_OBJ) {
      p = (uint32_t*)g_dev_arena->take(w * 4, s);
      borrowed = true;  // the arena owns it
    } else {
      if (g_mem_acct) {
        g_mem_acct->charge((int64_t)(w * 4));
        acct = g_mem_acct;
      }
      const cudaError_t e = cudaMallocAsync((void**)&p, w * 4, s);
      if (e != cudaSuccess) {
        cudaGetLastError();
        if (acct) acct->refund((int64_t)(w * 4));
        acct = nullptr;
        p = nullptr;
        throw Error(e == cudaErrorMemoryAllocation ? LG_ERR_OOM : LG_ERR_CUDA,
                    std::string("device allocation of ") + std::to_string(w * 4) + " bytes: " + cudaGetErrorString(e));
      }
    }
  }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept { *this = std::move(o); }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; words = o.words; st = o.st; borrowed = o.borrowed; acct = o.acct;
      o.p = nullptr; o.words = 0; o.acct = nullptr;
    }
    return *this;
  }
  ~DBuf() { release(); }
  void release() {
    if (p && !borrowed) {
      cudaFreeAsync(p, st);
      if (acct) acct->refund((int64_t)(words * 4));
    }
    p = nullptr;
    words = 0;
    acct = nullptr;
  }
};
using DBufP = std::shared_ptr<DBuf>;

// words [off, off + words) of `backing` as a buffer of its own; it keeps the
// backing alive.  Lets one allocation serve many groups or modules.
inline DBufP dbuf_slice(const DBufP& backing, size_t off, size_t words) {
  struct View {
    DBufP backing;
    DBuf v;
  };
  auto h = std::make_shared<View>();
  h->backing = backing;
  h->v.p = backing->p + off;
  h->v.words = words;
  h->v.st = backing->st;
  h->v.borrowed = true;
  return DBufP(h, &h->v);
}

struct ProgCache;  // compiled bytecode of one program (prover.cuh)

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // Work that overlaps a host wait on `stream` (the DEEP denominators while
  // the host hashes the claimed values): forked after fork_ev, joined back
  // through join_ev.
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  // A host witness's columns that the first commitment does not take go up
  // on `side` after the others, while round 0 runs; upload_ev marks the end.
  cudaEvent_t upload_ev = nullptr;
  DevArena dev_arena;            // prove-scoped small device buffers
  MemAcct mem;                   // device bytes this context holds (lg_ctx_mem_usage)
  std::map<int, DBufP> tw;       // log n -> w_n^j, j < n
  std::map<int, DBufP> tw16;     // log n -> the radix-16 passes' twiddle tables (tw16 layout, ntt16.cuh)
  std::map<int, DBufP> tw_split; // log n -> w_n's powers as two small Shoup tables (split_powers)
  std::map<int, DBufP> gpow;     // log n -> g^k, k < n
  std::map<int, DBufP> ginvpow;  // log n -> g^-k, k < n
  std::map<int, DBufP> cshift;   // log n -> (g w_4n^c)^k, k < n, for c = 0..3 (4 tables back to back)
  // Program-constant device data kept across proves: Lagrange columns
  // (log n, row) -> values and coefficients, and the compiled bytecode of the
  // most recently proven programs (most recent first).
  std::map<std::pair<uint32_t, uint32_t>, DBufP> lagrange_vals, lagrange_coef;
  std::list<std::shared_ptr<ProgCache>> programs;
  static constexpr size_t MAX_PROGRAMS = 8;
  std::string err;
  uint32_t* pinned = nullptr;    // host staging
  size_t pinned_words = 0;
  int sm_count = 148;

  // Timer marks (lg_timer_mark) and the optional per-kernel event profiler:
  // events recorded on this context's stream around selected launches, with
  // the algorithmic bytes and Poseidon2 permutations of each launch.
  cudaEvent_t marks[16] = {};
  struct KRec { const char* name; cudaEvent_t a, b; double bytes, perms; size_t phase; };  // phase: index of the prove phase it ran in
  bool profiling = false;
  std::vector<KRec> recs;
  std::vector<cudaEvent_t> event_pool;
  size_t event_next = 0;
  cudaEvent_t pooled_event() {
    if (event_next == event_pool.size()) {
      cudaEvent_t e;
      LG_CK(cudaEventCreate(&e));
      event_pool.push_back(e);
    }
    return event_pool[event_next++];
  }
  // Host wall time per prove phase (milliseconds), recorded when profiling.
  std::vector<uint8_t> proof_buf;  // encoding of the last proof (Writer target)
  std::vector<std::pair<std::string, double>> phases;
  std::chrono::steady_clock::time_point phase_t0;
  void phase_start() { phase_t0 = std::chrono::steady_clock::now(); phases.clear(); }
  void phase(const char* name) {
    if (!profiling) return;
    auto now = std::chrono::steady_clock::now();
    phases.emplace_back(name, std::chrono::duration<double, std::milli>(now - phase_t0).count());
    phase_t0 = now;
  }
  template <class F> void timed(const char* name, double bytes, double perms, F launch, cudaStream_t on = nullptr) {
    if (!profiling) { launch(); return; }
    if (!on) on = stream;
    KRec r{name, pooled_event(), pooled_event(), bytes, perms, phases.size()};
    LG_CK(cudaEventRecord(r.a, on));
    launch();
    LG_CK(cudaEventRecord(r.b, on));
    recs.push_back(r);
  }

  const uint32_t* twiddles(int logn) {
    auto it = tw.find(logn);
    if (it != tw.end()) return it->second->p;
    size_t n = (size_t)1 << logn;
    ArenaScope cached(nullptr);  // kept across proves: never from the arena
    auto b = std::make_shared<DBuf>(n, stream);
    k_fill_powers<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(b->p, n, root_of_unity_mont(logn), MONT_ONE);
    LG_LAUNCH();
    tw[logn] = b;
    return b->p;
  }
  // Twiddles of the radix-16 passes for 2^logn points (4 <= logn), pass by
  // pass in the tw16 layout of ntt16.cuh (canonical words, then their Shoup
  // companions); built on the host once per size.
  const uint32_t* twiddles16(int logn) {
    auto it = tw16.find(logn);
    if (it != tw16.end()) return it->second->p;
    const uint32_t n = 1u << logn;
    std::vector<uint32_t> pw(n);
    const uint32_t w = root_of_unity_mont(logn);
    pw[0] = MONT_ONE;
    for (uint32_t k = 1; k < n; k++) pw[k] = mul(pw[k - 1], w);
    const uint32_t W = tw16_words(logn);  // canonical twiddles, then their Shoup companions
    std::vector<uint32_t> tab(2 * (size_t)W, 0);
    for (int dif = 0; dif < 2; dif++)
      for (int invd = 0; invd < 2; invd++)
        for (int p = 0; p < pass_count(logn); p++) {
          int lo = 0, s_lo = 0, s_hi = 0;
          if (dif) pass_plan<true>(p, logn, lo, s_lo, s_hi);
          else pass_plan<false>(p, logn, lo, s_lo, s_hi);
          const uint32_t base = tw16_pass_offset(logn, dif != 0, invd != 0, p);
          for (int st = s_lo; st <= s_hi; st++) {
            const uint32_t m = 1u << (st - lo), off = base + tw16_stage_offset(s_lo, st);
            for (uint32_t tl = 0; tl < (1u << lo); tl++)
              for (uint32_t rl = 0; rl < m; rl++) {
                const uint32_t e = ((tl + (rl << lo)) << (logn - st - 1)) & (n - 1);
                const uint32_t wc = from_mont(pw[invd ? (n - e) & (n - 1) : e]);
                tab[off + tl * m + rl] = wc;
                tab[W + off + tl * m + rl] = shoup(wc);
              }
          }
        }
    ArenaScope cached(nullptr);  // kept across proves: never from the arena
    auto b = std::make_shared<DBuf>(tab.size(), stream);
    LG_CK(cudaMemcpyAsync(b->p, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, stream));
    LG_CK(cudaStreamSynchronize(stream));  // the host table goes out of scope
    tw16[logn] = b;
    return b->p;
  }
  // Powers of w = w_{2^logw} (logw > 11) for mul_split (ntt_large.cuh):
  // 2^11 pairs (w^i canonical, its Shoup companion), then 2^(logw - 11)
  // pairs for w^(2^11 i); built on the host once per size.
  const uint2* split_powers(int logw) {
    auto it = tw_split.find(logw);
    if (it != tw_split.end()) return reinterpret_cast<const uint2*>(it->second->p);
    if (logw <= 11 || logw > 30) throw Error(LG_ERR_INVALID, "split powers of an unsupported order");
    const uint32_t nlo = 1u << 11, nhi = 1u << (logw - 11);
    std::vector<uint32_t> tab(2 * (size_t)(nlo + nhi));
    const uint32_t w = root_of_unity_mont(logw);
    uint32_t x = MONT_ONE;
    for (uint32_t i = 0; i < nlo; i++) {
      tab[2 * i] = from_mont(x);
      tab[2 * i + 1] = shoup(tab[2 * i]);
      x = mul(x, w);
    }
    const uint32_t step = x;  // w^(2^11)
    x = MONT_ONE;
    for (uint32_t i = 0; i < nhi; i++) {
      tab[2 * (nlo + i)] = from_mont(x);
      tab[2 * (nlo + i) + 1] = shoup(tab[2 * (nlo + i)]);
      x = mul(x, step);
    }
    ArenaScope cached(nullptr);  // kept across proves: never from the arena
    auto b = std::make_shared<DBuf>(tab.size(), stream);
    LG_CK(cudaMemcpyAsync(b->p, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, stream));
    LG_CK(cudaStreamSynchronize(stream));  // the host table goes out of scope
    tw_split[logw] = b;
    return reinterpret_cast<const uint2*>(b->p);
  }
  // the table a transform kernel takes: tw16 for the radix-16 passes, the
  // plain powers below 16 points (radix-2 stages)
  const uint32_t* ntt_twiddles(int logn) { return logn >= 4 ? twiddles16(logn) : twiddles(logn); }
  const uint32_t* gpowers(int logn, bool inverse) {
    auto& m = inverse ? ginvpow : gpow;
    auto it = m.find(logn);
    if (it != m.end()) return it->second->p;
    size_t n = (size_t)1 << logn;
    ArenaScope cached(nullptr);  // kept across proves: never from the arena
    auto b = std::make_shared<DBuf>(n, stream);
    uint32_t g = to_mont(3);
    if (inverse) g = inv(g);
    k_fill_powers<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(b->p, n, g, MONT_ONE);
    LG_LAUNCH();
    m[logn] = b;
    return b->p;
  }
  // Coset shifts of the quotient cosets g w_4n^c <w_n>: (g w_4n^c)^k, k < n,
  // c = 0..3, one table after another.
  const uint32_t* coset_shifts(int logn) {
    auto it = cshift.find(logn);
    if (it != cshift.end()) return it->second->p;
    size_t n = (size_t)1 << logn;
    ArenaScope cached(nullptr);  // kept across proves: never from the arena
    auto b = std::make_shared<DBuf>(4 * n, stream);
    const uint32_t w4 = root_of_unity_mont(logn + 2);
    for (uint32_t cc = 0; cc < 4; cc++) {
      const uint32_t s = mul(to_mont(3), mont_pow(w4, cc));
      k_fill_powers<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(b->p + cc * n, n, s, MONT_ONE);
      LG_LAUNCH();
    }
    cshift[logn] = b;
    return b->p;
  }
  uint32_t* host_staging(size_t words) {
    if (words > pinned_words) {
      if (pinned) cudaFreeHost(pinned);
      pinned = nullptr;
      size_t w = std::max(words, (size_t)1 << 20);
      LG_CK(cudaMallocHost((void**)&pinned, w * 4));
      pinned_words = w;
    }
    return pinned;
  }
  void d2h(uint32_t* host, const uint32_t* dev, size_t words) {
    LG_CK(cudaMemcpyAsync(host, dev, words * 4, cudaMemcpyDeviceToHost, stream));
    LG_CK(cudaStreamSynchronize(stream));
  }
  // Small uploads (pointer tables, job descriptors, bytecode) go through a
  // pinned arena so the copy is asynchronous and the host can run ahead of
  // the device.  The arena restarts when the stream is idle (arena_reset at
  // the start of every call) or, when full, after a stream synchronize.
  uint8_t* arena = nullptr;
  size_t arena_cap = 0, arena_off = 0;
  void arena_reset() { arena_off = 0; }
  void h2d(uint32_t* dev, const void* host, size_t bytes) {
    size_t need = (bytes + 255) & ~(size_t)255;
    if (arena_off + need > arena_cap) {
      LG_CK(cudaStreamSynchronize(stream));
      if (need > arena_cap) {
        if (arena) cudaFreeHost(arena);
        arena = nullptr;
        arena_cap = std::max(need, (size_t)64 << 20);
        LG_CK(cudaMallocHost((void**)&arena, arena_cap));
      }
      arena_off = 0;
    }
    uint8_t* p = arena + arena_off;
    memcpy(p, host, bytes);
    arena_off += need;
    LG_CK(cudaMemcpyAsync(dev, p, bytes, cudaMemcpyHostToDevice, stream));
  }
  // One launch per phase over all groups / modules of a size (true), or one
  // launch per group / module (false, the plain per-kernel prover).
  bool batched = true;
  // Leaf hashing: 0 = choose by the amount of parallelism, 1 = one thread per
  // permutation, 6 = six lanes per permutation.
  int leaf_mapping = 0;
  // Launch-shape choices (lg_ctx_set_tuning, set by the autotuner); proofs do
  // not depend on them.  Defaults measured on B200.
  struct Tuning {
    uint32_t p2_leaf_min_per_sm = 128;  // one thread per leaf / injection chain from this many per SM
    uint32_t p2_node_min_per_sm = 512;  // one thread per node of a Merkle level from this many per SM
    uint32_t p2_inject_min_per_sm = 128;  // one thread per injection chain from this many per SM
    uint32_t merkle_tail = 32;          // levels narrower than this run in one block
    uint32_t merkle_subtree = 16;       // nodes a block reduces to one in the levels above (0: a launch per level)
    uint32_t inject_block = 32;         // threads per block, one-thread injection chains
    uint32_t leaf_block = 128;          // threads per block, one-thread leaf hashing
    uint32_t lde_split = 1;             // LDE as an inverse launch plus one block per (lane, coset)
    uint32_t lde_fwd_threads = 512;     // threads per block of the coset transforms (split LDE)
    uint32_t quotient_jit = 1;          // constraint bytecode (quotient, grand-product ratios) as compiled kernels (0: interpreter)
    uint32_t upload_split = 1;          // host witness: round 0's columns first, the rest on the side stream while
                                        // round 0 runs (0: every column before the prove starts)
    uint32_t fri_tail_leaves = 0;       // FRI rounds whose layer tree has at most this many leaves: one block (0: none;
                                        // 512 measured 14.09 ms against 13.65 ms per 40 x 2^14 prove)
  } tune;
};

// ---------------------------------------------------------------- program
// Flat descriptor; the format is documented in include/loom_gpu.h.
enum { OP_COL = 0, OP_COIN = 1, OP_CONST = 2, OP_ADD = 3, OP_SUB = 4, OP_MUL = 5, OP_EXPAVG = 6, OP_EXPVAL = 7 };
enum { KIND_WITNESS = 0, KIND_STEP = 1, KIND_LAGRANGE = 2, KIND_SETUP = 3 };
enum { STEP_GP = 0, STEP_MULT = 1, STEP_LOGUP = 2, STEP_RATIO = 3, STEP_MULTW = 4 };
inline bool exposes(uint32_t step_type) { return step_type == STEP_LOGUP || step_type == STEP_RATIO; }
inline bool is_binary(uint32_t op) { return op == OP_ADD || op == OP_SUB || op == OP_MUL; }
struct Module { uint32_t log_n; std::string name; std::vector<uint32_t> rels; };
struct Column { std::string name; uint32_t module, field, kind; int32_t param; };
struct Node { uint32_t op, a, b; };
struct Step {
  uint32_t type, round, module = 0, num = 0, den = 0, out = 0;
  std::vector<uint32_t> src, tgt, outs;  // lookup multiplicities (type 4: `width` nodes per table)
  uint32_t width = 1, flags = 0;         // type 4: tuple width; bit 0 source selectors, bit 1 target selectors
  std::vector<uint32_t> sel_s, sel_t;    // type 4 selectors
  std::vector<uint32_t> e, m;            // cyclic logup: fractions m[k] / e[k]
  uint32_t exposed = 0;                  // cyclic logup / running ratio: index of its exposed value
};
struct Program {
  uint32_t n_rounds = 0;
  std::vector<Module> modules;
  std::vector<Column> columns;
  std::vector<Node> nodes;
  std::vector<Step> steps;
  std::vector<std::vector<uint32_t>> staged;
};

inline Program parse_program(const uint32_t* w, size_t n) {
  size_t pos = 0;
  auto rd = [&]() -> uint32_t {
    if (pos >= n) throw Error(LG_ERR_INVALID, "program descriptor truncated");
    return w[pos++];
  };
  auto rds = [&]() {
    uint32_t len = rd();
    if (len > (n - pos) * 4) throw Error(LG_ERR_INVALID, "program descriptor: bad string length");
    std::string s(len, '\0');
    for (uint32_t i = 0; i < len; i += 4) {
      uint32_t x = rd();
      for (uint32_t j = 0; j < 4 && i + j < len; j++) s[i + j] = (char)((x >> (8 * j)) & 0xff);
    }
    return s;
  };
  Program p;
  if (rd() != 0x3150474Cu) throw Error(LG_ERR_INVALID, "program descriptor: bad magic");
  p.n_rounds = rd();
  uint32_t nm = rd(), nc = rd(), nn = rd(), ns = rd();
  if (p.n_rounds == 0) throw Error(LG_ERR_INVALID, "program descriptor: no rounds");
  for (uint32_t i = 0; i < nm; i++) {
    Module m;
    m.log_n = rd();
    if (m.log_n < 1 || m.log_n > 22) throw Error(LG_ERR_INVALID, "module size out of range (2 .. 2^22 rows)");
    m.name = rds();
    uint32_t nr = rd();
    for (uint32_t k = 0; k < nr; k++) m.rels.push_back(rd());
    p.modules.push_back(m);
  }
  for (uint32_t i = 0; i < nc; i++) {
    Column c;
    c.name = rds();
    c.module = rd(); c.field = rd(); c.kind = rd(); c.param = (int32_t)rd();
    if (c.module >= nm || c.field > 1 || c.kind > KIND_SETUP) throw Error(LG_ERR_INVALID, "bad column " + c.name);
    p.columns.push_back(c);
  }
  for (uint32_t i = 0; i < nn; i++) {
    Node x{rd(), rd(), rd()};
    if (x.op > OP_EXPVAL) throw Error(LG_ERR_INVALID, "bad node op");
    if (is_binary(x.op) && (x.a >= i || x.b >= i)) throw Error(LG_ERR_INVALID, "node children must precede parents");
    if (x.op == OP_COL && x.a >= nc) throw Error(LG_ERR_INVALID, "node column out of range");
    if (x.op == OP_COIN && x.a >= p.n_rounds) throw Error(LG_ERR_INVALID, "node coin out of range");
    p.nodes.push_back(x);
  }
  uint32_t n_exposed = 0;
  auto node = [&]() {
    uint32_t v = rd();
    if (v >= nn) throw Error(LG_ERR_INVALID, "step node out of range");
    return v;
  };
  auto column = [&]() {
    uint32_t v = rd();
    if (v >= nc) throw Error(LG_ERR_INVALID, "step column out of range");
    return v;
  };
  for (uint32_t i = 0; i < ns; i++) {
    Step s;
    s.type = rd();
    s.round = rd();
    if (s.type == STEP_GP || s.type == STEP_RATIO) {
      s.module = rd();
      s.num = node();
      s.den = node();
      s.out = column();
      if (s.type == STEP_RATIO) s.exposed = n_exposed++;
    } else if (s.type == STEP_MULT) {
      uint32_t a = rd(), b = rd();
      if (!a || !b || a > 4096 || b > 4096) throw Error(LG_ERR_INVALID, "bad multiplicity step");
      for (uint32_t k = 0; k < a; k++) s.src.push_back(node());
      for (uint32_t k = 0; k < b; k++) s.tgt.push_back(node());
      for (uint32_t k = 0; k < b; k++) s.outs.push_back(column());
    } else if (s.type == STEP_MULTW) {
      s.width = rd();
      uint32_t a = rd(), b = rd();
      s.flags = rd();
      if (!s.width || s.width > 8 || !a || !b || a > 4096 || b > 4096 || s.flags > 3)
        throw Error(LG_ERR_INVALID, "bad tuple multiplicity step");
      if (s.flags & 1) for (uint32_t k = 0; k < a; k++) s.sel_s.push_back(node());
      if (s.flags & 2) for (uint32_t k = 0; k < b; k++) s.sel_t.push_back(node());
      for (uint32_t k = 0; k < a * s.width; k++) s.src.push_back(node());
      for (uint32_t k = 0; k < b * s.width; k++) s.tgt.push_back(node());
      for (uint32_t k = 0; k < b; k++) s.outs.push_back(column());
    } else if (s.type == STEP_LOGUP) {
      s.module = rd();
      s.out = column();
      uint32_t t = rd();
      if (!t || t > 16) throw Error(LG_ERR_INVALID, "bad logup step");
      for (uint32_t k = 0; k < t; k++) {
        s.e.push_back(node());
        s.m.push_back(node());
      }
      s.exposed = n_exposed++;
    } else {
      throw Error(LG_ERR_INVALID, "unknown step type");
    }
    if (s.round >= p.n_rounds || s.module >= nm) throw Error(LG_ERR_INVALID, "bad step");
    p.steps.push_back(s);
  }
  for (const Node& x : p.nodes)
    if ((x.op == OP_EXPAVG || x.op == OP_EXPVAL) && x.a >= n_exposed)
      throw Error(LG_ERR_INVALID, "exposed value out of range");
  for (uint32_t r = 0; r < p.n_rounds; r++) {
    uint32_t k = rd();
    std::vector<uint32_t> v;
    for (uint32_t i = 0; i < k; i++) {
      uint32_t c = rd();
      if (c >= nc) throw Error(LG_ERR_INVALID, "staged column out of range");
      v.push_back(c);
    }
    p.staged.push_back(v);
  }
  for (auto& m : p.modules)
    for (uint32_t r : m.rels)
      if (r >= nn) throw Error(LG_ERR_INVALID, "relation root out of range");
  return p;
}

// ---------------------------------------------------------------- transcript
inline std::vector<uint32_t> string_to_elements(uint32_t tag, const std::string& s) {
  std::vector<uint32_t> r = {to_mont(tag), to_mont((uint32_t)s.size())};
  for (size_t i = 0; i < s.size(); i += 3) {
    uint32_t limb = 0;
    for (size_t j = 0; j < 3 && i + j < s.size(); j++) limb |= (uint32_t)(uint8_t)s[i + j] << (8 * j);
    r.push_back(to_mont(limb));
  }
  return r;
}

struct Digest { uint32_t v[8]; };

struct Transcript {
  // name_el: the name's field elements (string_to_elements), made once when
  // the challenge is declared
  struct Ch { std::string name; std::vector<uint32_t> name_el, bindings; Digest value; bool done = false; };
  std::vector<Ch> chs;
  std::map<std::string, size_t> index;
  void add(const std::string& n) {
    if (index.count(n)) throw Error(LG_ERR_INVALID, "duplicate challenge " + n);
    index[n] = chs.size();
    Ch c;
    c.name = n;
    c.name_el = string_to_elements(0x46534944u, n);
    chs.push_back(std::move(c));
  }
  void bind(const std::string& n, const uint32_t* v, size_t len) {
    auto it = index.find(n);
    if (it == index.end()) throw Error(LG_ERR_INVALID, "unknown challenge " + n);
    if (chs[it->second].done) throw Error(LG_ERR_INVALID, "challenge already computed " + n);
    chs[it->second].bindings.insert(chs[it->second].bindings.end(), v, v + len);
  }
  // What challenge n will hash, as far as the host has it: the name's
  // elements, whether a previous challenge exists and whether the host has
  // computed it (then its digest), and the bindings so far.
  struct Known { std::vector<uint32_t> name; bool has_prev = false, prev_done = false; Digest prev{}; std::vector<uint32_t> binds; };
  Known known(const std::string& n) const {
    auto it = index.find(n);
    if (it == index.end()) throw Error(LG_ERR_INVALID, "unknown challenge " + n);
    const size_t i = it->second;
    Known k;
    k.name = chs[i].name_el;
    if (i) {
      k.has_prev = true;
      k.prev_done = chs[i - 1].done;
      if (k.prev_done) k.prev = chs[i - 1].value;
    }
    k.binds = chs[i].bindings;
    return k;
  }
  Digest compute(const std::string& n) {
    auto it = index.find(n);
    if (it == index.end()) throw Error(LG_ERR_INVALID, "unknown challenge " + n);
    return compute_at(it->second);
  }
  // By position in declaration order (a long chain such as the query
  // challenges, without a lookup per step).
  size_t at(const std::string& n) const {
    auto it = index.find(n);
    if (it == index.end()) throw Error(LG_ERR_INVALID, "unknown challenge " + n);
    return it->second;
  }
  void bind_at(size_t i, const uint32_t* v, size_t len) {
    if (chs.at(i).done) throw Error(LG_ERR_INVALID, "challenge already computed " + chs[i].name);
    chs[i].bindings.insert(chs[i].bindings.end(), v, v + len);
  }
  Digest compute_at(size_t i) {
    Ch& ch = chs.at(i);
    if (ch.done) return ch.value;
    HostSponge h;
    for (uint32_t x : ch.name_el) h.write(x);
    if (i) {
      if (!chs[i - 1].done) throw Error(LG_ERR_INVALID, "previous challenge not computed for " + ch.name);
      for (int k = 0; k < 8; k++) h.write(chs[i - 1].value.v[k]);
    }
    for (uint32_t x : ch.bindings) h.write(x);
    h.sum(ch.value.v);
    ch.done = true;
    return ch.value;
  }
};
inline E6 digest_e6(const Digest& d) { E6 r; for (int i = 0; i < 6; i++) r.c[i] = d.v[i]; return r; }

// ---------------------------------------------------------------- proof writer
// Canonical encoding: 4-byte big-endian words, field elements canonical.
// `el*` take Montgomery words; `raw*` take words already canonical.
// Appends the proof encoding straight into the caller's output buffer while
// it fits; past its end, moves what it has to `spill` (a context-owned buffer
// reused from proof to proof, so its pages are touched once) and goes on
// there.
struct Writer {
  std::vector<uint8_t>& spill;
  uint8_t* p;
  size_t cap, off = 0;
  bool external;
  Writer(std::vector<uint8_t>& spill_buf, uint8_t* out, size_t out_cap) : spill(spill_buf) {
    external = out && out_cap;
    p = external ? out : spill.data();
    cap = external ? out_cap : spill.size();
  }
  void reserve(size_t bytes) {
    if (off + bytes <= cap) return;
    size_t want = std::max(off + bytes, 2 * off + ((size_t)1 << 20));
    if (spill.size() < want) spill.resize(want);
    if (external) memcpy(spill.data(), p, off);
    external = false;
    p = spill.data();
    cap = spill.size();
  }
  // size hint for the spill buffer (no effect while writing to the caller's)
  void expect(size_t bytes) { if (!external) reserve(bytes); }
  void put(uint32_t x) {
    reserve(4);
    uint32_t be = __builtin_bswap32(x);
    memcpy(p + off, &be, 4);
    off += 4;
  }
  void u32(uint32_t x) { put(x); }
  void el(uint32_t m) { put(from_mont(m)); }
  void e6(const E6& x) { for (int i = 0; i < 6; i++) el(x.c[i]); }
  void e6w(const uint32_t* w) { for (int i = 0; i < 6; i++) el(w[i]); }
  void dg(const Digest& d) { for (int i = 0; i < 8; i++) el(d.v[i]); }
  void dgw(const uint32_t* w) { for (int i = 0; i < 8; i++) el(w[i]); }
  void raw(uint32_t canonical) { put(canonical); }
  void raww(const uint32_t* w, size_t n) {
    reserve(4 * n);
    uint8_t* q = p + off;
    for (size_t i = 0; i < n; i++) {
      uint32_t be = __builtin_bswap32(w[i]);
      memcpy(q + 4 * i, &be, 4);
    }
    off += 4 * n;
  }
  // n bytes at the current offset, filled by the caller (a copy that lands
  // later); only while writing to the caller's buffer, which must hold them
  uint8_t* claim(size_t n) {
    if (!external || off + n > cap) throw Error(LG_ERR_INVALID, "proof writer: claimed bytes outside the caller's buffer");
    uint8_t* q = p + off;
    off += n;
    return q;
  }
  // words already in proof encoding (big-endian canonical bytes); large
  // blocks (the per-query sections, megabytes) are copied by four threads
  void bytes(const uint32_t* be, size_t n) {
    reserve(4 * n);
    const size_t len = 4 * n;
    if (len < ((size_t)2 << 20)) {
      memcpy(p + off, be, len);
    } else {
      const size_t parts = 4, step = (len / parts + 63) & ~(size_t)63;
      std::vector<std::thread> th;
      const uint8_t* src = reinterpret_cast<const uint8_t*>(be);
      for (size_t k = 1; k < parts; k++) {
        const size_t a = std::min(len, k * step), b = std::min(len, (k + 1) * step);
        if (a < b) th.emplace_back([=] { memcpy(p + off + a, src + a, b - a); });
      }
      memcpy(p + off, src, std::min(len, step));
      for (auto& t : th) t.join();
    }
    off += len;
  }
  void str(const std::string& s) {
    put((uint32_t)s.size());
    reserve(s.size());
    memcpy(p + off, s.data(), s.size());
    off += s.size();
  }
  size_t length() const { return off; }
  bool in_caller_buffer() const { return external; }
};

}  // namespace lg
