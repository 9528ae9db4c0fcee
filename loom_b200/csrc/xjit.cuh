// The constraint bytecode (XCode below, XInst in kernels.cuh) of the quotient
// and of the grand products' ratios compiled to kernels of their own at run time.  The interpreter (k_quotient_eval) keeps
// its register file in shared memory (6 words per register per thread, up
// to 72 KB per block) and decodes every instruction per row; the generated
// kernel names every register word as a local, so the compiler allocates
// real registers and the instruction stream is straight-line code.  The
// semantics are the interpreter's word for word: a base write sets word 0
// of its register and leaves the other five as they were, a base read
// takes word 0.
//
// The run-time compiler (NVRTC) is loaded with dlopen and the driver's
// module calls come through cudaGetDriverEntryPoint, so the library links
// neither; where either is missing, or a program is too long, the
// interpreter runs instead.  Kernels are cached per device and source.
#pragma once
#include <cuda.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <array>
#include <mutex>
#include <sstream>

#include "host.cuh"

namespace lg {

// Register bytecode of one expression (compile_expr, prover.cuh).
struct XCode { std::vector<XInst> code; uint32_t n_regs = 0, result = 0, result_ext = 0; };

// Job of a generated kernel (the QJob fields it needs); the generated
// source declares the same struct.
struct QxJob { const uint32_t* cv; uint32_t* qv; int logn; uint32_t zinv[4]; };
static_assert(sizeof(QxJob) == 40, "QxJob layout is shared with the generated source");
constexpr uint32_t XJIT_MAX_INST = 4096;

inline const char* xjit_field_src() {
  static const char* s =
#include "field_src.inc"
      ;
  return s;
}

// Statements evaluating one bytecode program for row j into `o` (locals
// named with prefix `pfx`); lane(l, shift) is the expression reading column
// lane l at row (j + shift) mod n; `reg` holds the expression of every
// register word (carried from a program run before in the same register
// file, as the interpreter carries them).  Returns the result as an E6
// expression.
using XRegs = std::vector<std::array<std::string, 6>>;
inline XRegs xjit_regs(uint32_t n) {
  XRegs r(std::max<uint32_t>(n, 1));
  for (auto& w : r) w.fill("0u");
  return r;
}
template <class LaneExpr>
inline std::string xjit_body(std::ostringstream& o, const XCode& xc, const std::string& pfx, LaneExpr lane, XRegs& reg) {
  if (reg.size() < xc.n_regs) throw Error(LG_ERR_INVALID, "bytecode: register file too small");
  auto e6lit = [&](uint32_t r) {
    std::string s = "E6{{";
    for (int w = 0; w < 6; w++) s += (w ? ", " : "") + reg[r][w];
    return s + "}}";
  };
  for (size_t i = 0; i < xc.code.size(); i++) {
    const XInst& in = xc.code[i];
    const std::string v = pfx + std::to_string(i);
    auto base = [&](const std::string& expr) {
      o << "  const uint32_t " << v << " = " << expr << ";\n";
      reg[in.d][0] = v;
    };
    auto ext = [&](const std::string& expr) {
      o << "  const E6 " << v << " = " << expr << ";\n";
      for (int w = 0; w < 6; w++) reg[in.d][w] = v + ".c[" + std::to_string(w) + "]";
    };
    const std::string a0 = reg[in.a][0], b0 = reg[in.b][0];
    switch (in.op) {
      case X_LOAD_B: base(lane(in.imm, in.shift)); break;
      case X_LOAD_E: {
        std::string s = "E6{{";
        for (int w = 0; w < 6; w++) s += (w ? ", " : "") + lane(in.imm + w, in.shift);
        ext(s + "}}");
        break;
      }
      case X_COIN: ext("coins[" + std::to_string(in.imm) + "]"); break;
      case X_CONST: base(std::to_string(in.imm) + "u"); break;
      case X_ADD_BB: base("add(" + a0 + ", " + b0 + ")"); break;
      case X_SUB_BB: base("sub(" + a0 + ", " + b0 + ")"); break;
      case X_MUL_BB: base("mul(" + a0 + ", " + b0 + ")"); break;
      case X_ADD_EE: ext("e6_add(" + e6lit(in.a) + ", " + e6lit(in.b) + ")"); break;
      case X_SUB_EE: ext("e6_sub(" + e6lit(in.a) + ", " + e6lit(in.b) + ")"); break;
      case X_MUL_EE: ext("e6_mul(" + e6lit(in.a) + ", " + e6lit(in.b) + ")"); break;
      case X_MUL_EB: ext("e6_mul_base(" + e6lit(in.a) + ", " + b0 + ")"); break;
      case X_ADD_EB: case X_SUB_EB: {
        std::string s = "E6{{" + std::string(in.op == X_ADD_EB ? "add(" : "sub(") + a0 + ", " + b0 + ")";
        for (int w = 1; w < 6; w++) s += ", " + reg[in.a][w];
        ext(s + "}}");
        break;
      }
      case X_SUB_BE: {
        std::string s = "E6{{sub(" + a0 + ", " + b0 + ")";
        for (int w = 1; w < 6; w++) s += ", neg(" + reg[in.b][w] + ")";
        ext(s + "}}");
        break;
      }
      default: throw Error(LG_ERR_INVALID, "bytecode: unknown instruction");
    }
  }
  return xc.result_ext ? e6lit(xc.result) : "e6_base(" + reg[xc.result][0] + ")";
}

// CUDA source of the quotient kernel of one bytecode program.
inline std::string xjit_source(const XCode& xc) {
  std::ostringstream o;
  o << "#include \"field.cuh\"\nusing namespace lg;\n"
       "struct QxJob { const uint32_t* cv; uint32_t* qv; int logn; uint32_t zinv[4]; };\n"
       "extern \"C\" __global__ void __launch_bounds__(128) lg_qx(const QxJob* jobs, const E6* coins) {\n"
       "  const QxJob J = jobs[blockIdx.z];\n"
       "  const uint32_t n = 1u << J.logn, c = blockIdx.y, m = n - 1;\n"
       "  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;\n"
       "  if (j >= n) return;\n"
       "  const uint64_t big = (uint64_t)n << 2;\n"
       "  const uint32_t* cv = J.cv + (uint64_t)c * n;\n";
  XRegs reg = xjit_regs(xc.n_regs);
  const std::string res = xjit_body(o, xc, "v", [](uint32_t l, int32_t shift) {
    return "cv[" + std::to_string(l) + "ull * big + ((j + " + std::to_string((uint32_t)shift) + "u) & m)]";
  }, reg);
  o << "  const E6 r = e6_mul_base(" << res << ", J.zinv[c]);\n";
  const int lw = xc.result_ext ? 6 : 1;
  for (int w = 0; w < lw; w++)
    o << "  J.qv[" << w << "ull * big + (uint64_t)c * n + j] = r.c[" << w << "];\n";
  o << "}\n";
  return o.str();
}

// Job of a compiled grand-product ratio kernel (GpJob's fields it needs).
struct GpxJob { const uint32_t* const* lanes; uint32_t* ratio; int logn; };
static_assert(sizeof(GpxJob) == 24, "GpxJob layout is shared with the generated source");

// CUDA source of a grand product's ratio num(j) / den(j) (k_gp_ratio).
inline std::string xjit_gp_source(const XCode& num, const XCode& den) {
  std::ostringstream o;
  o << "#include \"field.cuh\"\nusing namespace lg;\n"
       "struct GpxJob { const uint32_t* const* lanes; uint32_t* ratio; int logn; };\n"
       "extern \"C\" __global__ void __launch_bounds__(128) lg_gpx(const GpxJob* jobs, const E6* coins) {\n"
       "  const GpxJob J = jobs[blockIdx.y];\n"
       "  const uint32_t n = 1u << J.logn, m = n - 1;\n"
       "  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;\n"
       "  if (j >= n) return;\n"
       "  const uint32_t* const* lanes = J.lanes;\n";
  auto lane = [](uint32_t l, int32_t shift) {
    return "lanes[" + std::to_string(l) + "][(j + " + std::to_string((uint32_t)shift) + "u) & m]";
  };
  XRegs reg = xjit_regs(std::max(num.n_regs, den.n_regs));  // one register file, as the interpreter's
  const std::string a = xjit_body(o, num, "a", lane, reg);
  o << "  const E6 na = " << a << ";\n";
  const std::string b = xjit_body(o, den, "b", lane, reg);
  o << "  const E6 q = e6_mul(na, e6_inv(" << b << "));\n";
  for (int w = 0; w < 6; w++) o << "  J.ratio[" << w << "ull * n + j] = q.c[" << w << "];\n";
  o << "}\n";
  return o.str();
}

// NVRTC entry points (dlopen) and the driver's module calls.
struct XjitApi {
  bool ok = false;
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
  decltype(&cuModuleLoadData) load = nullptr;
  decltype(&cuModuleGetFunction) get = nullptr;
  decltype(&cuLaunchKernel) launch = nullptr;
};
inline const XjitApi& xjit_api() {
  static XjitApi a = [] {
    XjitApi r;
    void* h = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libnvrtc.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) return r;
    r.create = (decltype(r.create))dlsym(h, "nvrtcCreateProgram");
    r.compile = (decltype(r.compile))dlsym(h, "nvrtcCompileProgram");
    r.log_size = (decltype(r.log_size))dlsym(h, "nvrtcGetProgramLogSize");
    r.log = (decltype(r.log))dlsym(h, "nvrtcGetProgramLog");
    r.cubin_size = (decltype(r.cubin_size))dlsym(h, "nvrtcGetCUBINSize");
    r.cubin = (decltype(r.cubin))dlsym(h, "nvrtcGetCUBIN");
    r.destroy = (decltype(r.destroy))dlsym(h, "nvrtcDestroyProgram");
    auto entry = [](const char* name, void** fn) {
      cudaDriverEntryPointQueryResult q;
      return cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q) == cudaSuccess &&
             q == cudaDriverEntryPointSuccess && *fn;
    };
    void *l = nullptr, *g = nullptr, *k = nullptr;
    const bool drv = entry("cuModuleLoadData", &l) && entry("cuModuleGetFunction", &g) && entry("cuLaunchKernel", &k);
    cudaGetLastError();
    r.load = (decltype(r.load))l;
    r.get = (decltype(r.get))g;
    r.launch = (decltype(r.launch))k;
    r.ok = drv && r.create && r.compile && r.log_size && r.log && r.cubin_size && r.cubin && r.destroy;
    return r;
  }();
  return a;
}

inline std::atomic<uint64_t> g_xjit_compiled{0};
inline uint64_t xjit_compiled() { return g_xjit_compiled.load(); }

// The kernel `name` of source `src` on the current device (compiled on first
// use, then cached); null when it cannot be had (the interpreter runs).
inline CUfunction xjit_compile(const std::string& src, const char* name) {
  const XjitApi& api = xjit_api();
  if (!api.ok) return nullptr;
  int dev = 0;
  LG_CK(cudaGetDevice(&dev));
  static std::mutex mu;
  static std::map<std::pair<int, std::string>, CUfunction> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_pair(dev, src);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  CUfunction fn = nullptr;
  nvrtcProgram prog = nullptr;
  const char* hdr[] = {xjit_field_src()};
  const char* hname[] = {"field.cuh"};
  if (api.create(&prog, src.c_str(), "lg_x.cu", 1, hdr, hname) == NVRTC_SUCCESS) {
    const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device"};
    size_t sz = 0;
    if (api.compile(prog, 3, opts) == NVRTC_SUCCESS && api.cubin_size(prog, &sz) == NVRTC_SUCCESS && sz) {
      std::vector<char> bin(sz);
      CUmodule mod = nullptr;
      if (api.cubin(prog, bin.data()) == NVRTC_SUCCESS && api.load(&mod, bin.data()) == CUDA_SUCCESS &&
          api.get(&fn, mod, name) != CUDA_SUCCESS)
        fn = nullptr;
    }
    api.destroy(&prog);
  }
  cache[key] = fn;  // a failure is remembered too: the interpreter serves that program
  if (fn) g_xjit_compiled.fetch_add(1);
  return fn;
}
inline CUfunction xjit_quotient(const XCode& xc) {
  if (xc.code.empty() || xc.code.size() > XJIT_MAX_INST) return nullptr;
  return xjit_compile(xjit_source(xc), "lg_qx");
}
inline CUfunction xjit_gp(const XCode& num, const XCode& den) {
  if (num.code.empty() || den.code.empty() || num.code.size() + den.code.size() > XJIT_MAX_INST) return nullptr;
  return xjit_compile(xjit_gp_source(num, den), "lg_gpx");
}

inline void xjit_launch(CUfunction fn, dim3 grid, const void* jobs_d, const E6* coins_d, cudaStream_t s) {
  void* args[] = {(void*)&jobs_d, (void*)&coins_d};
  if (xjit_api().launch(fn, grid.x, grid.y, grid.z, 128, 1, 1, 0, (CUstream)s, args, nullptr) != CUDA_SUCCESS)
    throw Error(LG_ERR_CUDA, "launch of a compiled constraint kernel failed");
}

}  // namespace lg
