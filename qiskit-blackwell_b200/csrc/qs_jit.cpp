// qs_jit.cpp — runtime specialisation of tile passes (NVRTC, sm_100a).
//
// The tile-pass interpreter (qs_pass.cu) reads its program at run time: op
// dispatch, runtime register positions and moves between the register array
// and temporaries cost about as many issue slots as the arithmetic itself.
// A plan that runs on large states is instead compiled pass by pass into
// kernels of its own: register positions, swizzled shared-memory offsets,
// the op sequence and the coefficients (as exact hexadecimal float literals)
// are compile-time constants, and amplitudes are renamed instead of moved.
//
// The generator walks the same device program (DevPass / DevBlock / DevOp /
// coefficient pool) the interpreter executes and writes out the identical
// sequence of IEEE operations (the same fmaf / __fmul_rn chains, the same
// selects), so a specialised pass returns the interpreter's amplitudes bit
// for bit.  NVRTC and the driver API are opened with dlopen at first use; if
// either is missing or a compile fails, the plan stays on the interpreter.
#include "qs_api.h"
#include <cuda.h>
#include <nvrtc.h>
#include <dlfcn.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_map>

namespace {

// ------------------------------------------------------------ dlopen'd APIs
struct Api {
  bool nvrtc_ok = false, driver_ok = false;
  std::string why_nvrtc, why_driver;
  decltype(&nvrtcCreateProgram) CreateProgram = nullptr;
  decltype(&nvrtcCompileProgram) CompileProgram = nullptr;
  decltype(&nvrtcGetCUBINSize) GetCUBINSize = nullptr;
  decltype(&nvrtcGetCUBIN) GetCUBIN = nullptr;
  decltype(&nvrtcGetProgramLogSize) GetProgramLogSize = nullptr;
  decltype(&nvrtcGetProgramLog) GetProgramLog = nullptr;
  decltype(&nvrtcDestroyProgram) DestroyProgram = nullptr;
  decltype(&cuModuleLoadData) ModuleLoadData = nullptr;
  decltype(&cuModuleGetFunction) ModuleGetFunction = nullptr;
  decltype(&cuFuncSetAttribute) FuncSetAttribute = nullptr;
  decltype(&cuLaunchKernel) LaunchKernel = nullptr;
  decltype(&cuOccupancyMaxActiveBlocksPerMultiprocessor) Occupancy = nullptr;
  decltype(&cuTensorMapEncodeTiled) EncodeTiled = nullptr;  // optional: pipelined passes
};

Api& g_api = *new Api;  // never destroyed (background compiles may outlive main)
std::once_flag g_api_once;

template <class F>
bool sym(void* lib, const char* name, F& f) {
  f = reinterpret_cast<F>(dlsym(lib, name));
  return f != nullptr;
}

// NVRTC (the compiler, usable without a GPU) and the driver API (module
// loading and launches) are opened separately.
void load_api() {
  void* nv = nullptr;
  for (const char* n : {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"}) {
    nv = dlopen(n, RTLD_NOW | RTLD_LOCAL);
    if (nv) break;
  }
  if (!nv) {
    g_api.why_nvrtc = "libnvrtc.so.12 not found";
  } else if (sym(nv, "nvrtcCreateProgram", g_api.CreateProgram) &&
             sym(nv, "nvrtcCompileProgram", g_api.CompileProgram) &&
             sym(nv, "nvrtcGetCUBINSize", g_api.GetCUBINSize) && sym(nv, "nvrtcGetCUBIN", g_api.GetCUBIN) &&
             sym(nv, "nvrtcGetProgramLogSize", g_api.GetProgramLogSize) &&
             sym(nv, "nvrtcGetProgramLog", g_api.GetProgramLog) &&
             sym(nv, "nvrtcDestroyProgram", g_api.DestroyProgram)) {
    g_api.nvrtc_ok = true;
  } else {
    g_api.why_nvrtc = "an NVRTC entry point is missing";
  }
  void* cu = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
  if (!cu) {
    g_api.why_driver = "libcuda.so.1 not found";
  } else if (sym(cu, "cuModuleLoadData", g_api.ModuleLoadData) &&
             sym(cu, "cuModuleGetFunction", g_api.ModuleGetFunction) &&
             sym(cu, "cuFuncSetAttribute", g_api.FuncSetAttribute) &&
             sym(cu, "cuLaunchKernel", g_api.LaunchKernel) &&
             sym(cu, "cuOccupancyMaxActiveBlocksPerMultiprocessor", g_api.Occupancy)) {
    g_api.driver_ok = true;
    sym(cu, "cuTensorMapEncodeTiled", g_api.EncodeTiled);
  } else {
    g_api.why_driver = "a CUDA driver entry point is missing";
  }
}

// ------------------------------------------------------------ source text
// Device helpers: the same operations, in the same order, as qs_common.cuh's
// cfma2/cfma4 and qs_pass.cu's cmul / rotation / sign-flip code.
const char* kPrelude = R"(typedef unsigned long long u64;
typedef unsigned int u32;
__device__ __forceinline__ u32 phys(u32 i) { return i ^ ((((i >> 4) ^ (i >> 8) ^ (i >> 12)) & 7u) << 1); }
__device__ __forceinline__ u64 ins0(u64 x, int q) { const u64 lo = x & ((1ull << q) - 1ull); return ((x ^ lo) << 1) | lo; }
__device__ __forceinline__ u32 ins0w(u32 x, int q) { const u32 lo = x & ((1u << q) - 1u); return ((x ^ lo) << 1) | lo; }
__device__ __forceinline__ float2 cfma2(float2 g0, float2 a0, float2 g1, float2 a1) {
  float re = __fmul_rn(g0.x, a0.x); re = fmaf(-g0.y, a0.y, re); re = fmaf(g1.x, a1.x, re); re = fmaf(-g1.y, a1.y, re);
  float im = __fmul_rn(g0.x, a0.y); im = fmaf(g0.y, a0.x, im); im = fmaf(g1.x, a1.y, im); im = fmaf(g1.y, a1.x, im);
  return make_float2(re, im);
}
__device__ __forceinline__ float2 cfma4(float2 g0, float2 g1, float2 g2, float2 g3,
                                        float2 a0, float2 a1, float2 a2, float2 a3) {
  float re = __fmul_rn(g0.x, a0.x); re = fmaf(-g0.y, a0.y, re); re = fmaf(g1.x, a1.x, re); re = fmaf(-g1.y, a1.y, re);
  re = fmaf(g2.x, a2.x, re); re = fmaf(-g2.y, a2.y, re); re = fmaf(g3.x, a3.x, re); re = fmaf(-g3.y, a3.y, re);
  float im = __fmul_rn(g0.x, a0.y); im = fmaf(g0.y, a0.x, im); im = fmaf(g1.x, a1.y, im); im = fmaf(g1.y, a1.x, im);
  im = fmaf(g2.x, a2.y, im); im = fmaf(g2.y, a2.x, im); im = fmaf(g3.x, a3.y, im); im = fmaf(g3.y, a3.x, im);
  return make_float2(re, im);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -__fmul_rn(a.y, b.y)), fmaf(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 ry0(float co, float si, float2 a0, float2 a1) {
  return make_float2(fmaf(co, a0.x, -__fmul_rn(si, a1.x)), fmaf(co, a0.y, -__fmul_rn(si, a1.y)));
}
__device__ __forceinline__ float2 ry1(float co, float si, float2 a0, float2 a1) {
  return make_float2(fmaf(si, a0.x, __fmul_rn(co, a1.x)), fmaf(si, a0.y, __fmul_rn(co, a1.y)));
}
// Scaled rotations (DK_KRY) as packed FP32x2 FMAs: one instruction per
// output amplitude, lane results identical to the scalar fmaf.  t * a0 - a1
// is two scalar FMAs instead: the packed form has no negated addend, and the
// negation of a1 cost two FADDs on the FMA pipe besides the two cycles of the
// packed FMA (same bits either way: the negation is exact).
__device__ __forceinline__ float2 rta0(float t, float2 a0, float2 a1) { return __ffma2_rn(make_float2(-t, -t), a1, a0); }
__device__ __forceinline__ float2 rta1(float t, float2 a0, float2 a1) { return __ffma2_rn(make_float2(t, t), a0, a1); }
__device__ __forceinline__ float2 rtb0(float t, float2 a0, float2 a1) {
  return make_float2(fmaf(t, a0.x, -a1.x), fmaf(t, a0.y, -a1.y));
}
__device__ __forceinline__ float2 rtb1(float t, float2 a0, float2 a1) { return __ffma2_rn(make_float2(t, t), a1, a0); }
// The same four updates as two scalar FMAs (identical results lane by lane).
__device__ __forceinline__ float2 sta0(float t, float2 a0, float2 a1) { return make_float2(fmaf(-t, a1.x, a0.x), fmaf(-t, a1.y, a0.y)); }
__device__ __forceinline__ float2 sta1(float t, float2 a0, float2 a1) { return make_float2(fmaf(t, a0.x, a1.x), fmaf(t, a0.y, a1.y)); }
__device__ __forceinline__ float2 stb0(float t, float2 a0, float2 a1) { return make_float2(fmaf(t, a0.x, -a1.x), fmaf(t, a0.y, -a1.y)); }
__device__ __forceinline__ float2 stb1(float t, float2 a0, float2 a1) { return make_float2(fmaf(t, a1.x, a0.x), fmaf(t, a1.y, a0.y)); }
__device__ __forceinline__ float2 scl(float2 a, float f) { return make_float2(__fmul_rn(a.x, f), __fmul_rn(a.y, f)); }
__device__ __forceinline__ float2 sgnw(float2 t, u32 w) {
  return make_float2(__uint_as_float(__float_as_uint(t.x) ^ w), __uint_as_float(__float_as_uint(t.y) ^ w));
}
)";

// Exact float literal (hexadecimal significand).
std::string flit(float f) {
  if (f == 0.0f) return std::signbit(f) ? "(-0.0f)" : "0.0f";
  char buf[64];
  std::snprintf(buf, sizeof(buf), "(%af)", (double)f);
  return buf;
}
std::string c2(float2 v) { return "make_float2(" + flit(v.x) + ", " + flit(v.y) + ")"; }
uint64_t bits64(float2 f) {
  uint32_t lo, hi;
  std::memcpy(&lo, &f.x, 4);
  std::memcpy(&hi, &f.y, 4);
  return (uint64_t)lo | ((uint64_t)hi << 32);
}
uint32_t bits32(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
std::string mask_test(uint64_t gm, bool& used) {
  used = true;
  return "((gidx & " + std::to_string(gm) + "ull) == " + std::to_string(gm) + "ull)";
}

// Straight-line register block: amplitude j lives in the SSA value v[j].
struct Block {
  std::ostringstream o;
  std::vector<std::string> v;
  int fresh = 0;
  bool uses_g = false;  // an op reads the global amplitude index
  std::string name(const char* p) { return p + std::to_string(fresh++); }
  // v[j] := pred ? expr : v[j]   (pred "" = always)
  void set(int j, const std::string& expr, const std::string& pred) {
    const std::string n = name("a");
    if (pred.empty()) o << "      const float2 " << n << " = " << expr << ";\n";
    else o << "      const float2 " << n << " = " << pred << " ? " << expr << " : " << v[j] << ";\n";
    v[j] = n;
  }
};

// Threads per CTA: one register group per thread, at most 128 for R = 5
// blocks (QSIM_JIT_THREADS = 256 allows 256) and 256 otherwise.
// Rotation pairs emitted as packed FP32x2 FMAs, except every `n`-th pair as
// two scalar FMAs (QSIM_JIT_SCALAR_EVERY = n; 0 = all packed): a tuning knob
// for the balance between the FMA sub-pipes.  Results are identical.
int scalar_every() {
  static const int n = [] {
    const char* e = std::getenv("QSIM_JIT_SCALAR_EVERY");
    return e ? std::max(0, std::atoi(e)) : 0;
  }();
  return n;
}
std::string rot_fn(bool form_b, bool second, int pair_index) {
  const int n = scalar_every();
  const bool scalar = n > 0 && (pair_index % n) == 0;
  std::string f = scalar ? "st" : "rt";
  f += form_b ? "b" : "a";
  f += second ? "1(" : "0(";
  return f;
}

int pass_threads(int T, int R) {
  static const int cap5 = [] {
    const char* e = std::getenv("QSIM_JIT_THREADS");
    return (e && std::atoi(e) == 256) ? 256 : 128;
  }();
  return std::max(32, std::min(R >= 5 ? cap5 : 256, 1 << (T - R)));
}
int pass_smem(int T) { return (8 << T) + 2 * 128 * 8; }

void gen_block(Block& G, int R, const DevOp* ops, int ob, int oe, const float2* coef) {
  const int J = 1 << R;
  std::ostringstream& o = G.o;
  for (int oi = ob; oi < oe; ++oi) {
    const DevOp& op = ops[oi];
    const float2* c = coef + op.coef;
    std::string gp;  // "" = the global-control predicate is always true
    if (op.gc) {
      gp = G.name("gp");
      o << "      const bool " << gp << " = " << mask_test(op.gc, G.uses_g) << ";\n";
    }
    // false: a register control is unmet, the amplitudes are left unchanged
    auto active = [&](int j) { return (j & op.rc) == op.rc; };
    switch (op.kind) {
      case DK_U1:
      case DK_RY:
      case DK_X:
      case DK_Y: {
        const int A = op.t0;
        for (int j = 0; j < J; ++j) {
          if (((j >> A) & 1) || !active(j)) continue;
          const int k = j | (1 << A);
          const std::string a0 = G.v[j], a1 = G.v[k];
          if (op.kind == DK_U1) {
            G.set(j, "cfma2(" + c2(c[0]) + ", " + a0 + ", " + c2(c[1]) + ", " + a1 + ")", gp);
            G.set(k, "cfma2(" + c2(c[2]) + ", " + a0 + ", " + c2(c[3]) + ", " + a1 + ")", gp);
          } else if (op.kind == DK_RY) {
            const std::string cs = flit(c[0].x) + ", " + flit(c[0].y);
            G.set(j, "ry0(" + cs + ", " + a0 + ", " + a1 + ")", gp);
            G.set(k, "ry1(" + cs + ", " + a0 + ", " + a1 + ")", gp);
          } else if (op.kind == DK_X) {
            if (gp.empty()) {
              G.v[j] = a1;
              G.v[k] = a0;
            } else {
              G.set(j, a1, gp);
              G.set(k, a0, gp);
            }
          } else {
            G.set(j, "make_float2(" + a1 + ".y, -" + a1 + ".x)", gp);
            G.set(k, "make_float2(-" + a0 + ".y, " + a0 + ".x)", gp);
          }
        }
        break;
      }
      case DK_KRY:
      case DK_KU1: {
        for (int K = 0; K < R; ++K) {
          if (!((op.t0 >> K) & 1)) continue;
          int pair = 0;
          for (int j = 0; j < J; ++j) {
            if ((j >> K) & 1) continue;
            ++pair;
            const int k = j | (1 << K);
            const std::string a0 = G.v[j], a1 = G.v[k];
            if (op.kind == DK_KRY) {  // scaled rotation, form c[K].y (see DK_KRY)
              const std::string t = flit(c[K].x) + ", " + a0 + ", " + a1 + ")";
              const bool fb = c[K].y != 0.f;
              G.set(j, rot_fn(fb, false, pair) + t, "");
              G.set(k, rot_fn(fb, true, pair) + t, "");
            } else {
              const float2* g = c + 4 * K;
              G.set(j, "cfma2(" + c2(g[0]) + ", " + a0 + ", " + c2(g[1]) + ", " + a1 + ")", "");
              G.set(k, "cfma2(" + c2(g[2]) + ", " + a0 + ", " + c2(g[3]) + ", " + a1 + ")", "");
            }
          }
        }
        break;
      }
      case DK_SCALE:
        for (int j = 0; j < J; ++j) G.set(j, "scl(" + G.v[j] + ", " + flit(c[0].x) + ")", "");
        break;
      case DK_XRY: {  // parity rotation: pairs (j, j ^ (A|B)), coefficients by bit B
        const int A = op.t0, B = op.t1;
        int pair = 0;
        for (int j = 0; j < J; ++j) {
          if ((j >> A) & 1) continue;
          ++pair;
          const int k = j ^ ((1 << A) | (1 << B));
          const float2 tf = ((j >> B) & 1) ? c[1] : c[0];
          const std::string t = flit(tf.x) + ", " + G.v[j] + ", " + G.v[k] + ")";
          const bool fb = tf.y != 0.f;
          G.set(j, rot_fn(fb, false, pair) + t, "");
          G.set(k, rot_fn(fb, true, pair) + t, "");
        }
        break;
      }
      case DK_U2:
      case DK_CU2:
      case DK_SWAP: {
        const int A = op.t0, B = op.t1;
        for (int j = 0; j < J; ++j) {
          if ((j & ((1 << A) | (1 << B))) || !active(j)) continue;
          const int j1 = j | (1 << A), j2 = j | (1 << B), j3 = j1 | (1 << B);
          if (op.kind == DK_SWAP) {
            const std::string a = G.v[j1], b = G.v[j2];
            if (gp.empty()) {
              G.v[j1] = b;
              G.v[j2] = a;
            } else {
              G.set(j1, b, gp);
              G.set(j2, a, gp);
            }
            continue;
          }
          const std::string args = G.v[j] + ", " + G.v[j1] + ", " + G.v[j2] + ", " + G.v[j3] + ")";
          const int idx[4] = {j, j1, j2, j3};
          for (int r = 0; r < 4; ++r)
            G.set(idx[r], "cfma4(" + c2(c[4 * r]) + ", " + c2(c[4 * r + 1]) + ", " + c2(c[4 * r + 2]) + ", " +
                              c2(c[4 * r + 3]) + ", " + args, gp);
        }
        break;
      }
      case DK_DTAB: {
        // Layout (encode_dtab in qs_plan.cpp): [2^R table if rc&1]
        // [t0 group factors: mask, w][t1 sign terms: regmask, mask]
        // [d0 cross terms: regmask, mask, w].
        const bool table = op.rc & 1;
        const float2* p = c;
        const float2* Tt = p;
        if (table) p += J;
        const std::string f = G.name("f");
        if (op.t0) o << "      float " << f << "r = 1.f, " << f << "i = 0.f;\n";
        for (int k = 0; k < op.t0; ++k, p += 2) {
          const std::string wx = flit(p[1].x), wy = flit(p[1].y);
          o << "      if " << mask_test(bits64(p[0]), G.uses_g) << " { const float r_ = fmaf(" << f << "r, " << wx
            << ", -__fmul_rn(" << f << "i, " << wy << ")); " << f << "i = fmaf(" << f << "r, " << wy
            << ", __fmul_rn(" << f << "i, " << wx << ")); " << f << "r = r_; }\n";
        }
        // Sign terms: amplitude j is negated by the XOR of the predicates of
        // the terms whose register mask holds j.  Each distinct set of terms
        // gets one sign word per group; the word is XORed into the group
        // factor (or the table entry, or the amplitude) - the same bits the
        // generic kernel produces with its per-group mask.
        std::vector<uint64_t> rms;
        std::vector<std::string> sb;
        for (int k = 0; k < op.t1; ++k, p += 2) {
          rms.push_back(bits64(p[0]));
          sb.push_back(G.name("sb"));
          o << "      const u32 " << sb.back() << " = " << mask_test(bits64(p[1]), G.uses_g)
            << " ? 0x80000000u : 0u;\n";
        }
        if (rms.size() > 64) throw qs_error(QS_ERR_INVALID, "tile-pass specialisation: too many sign terms");
        std::map<uint64_t, std::string> word;  // term subset -> sign word
        auto subset = [&](int j) {
          uint64_t sub = 0;
          for (size_t k = 0; k < rms.size(); ++k)
            if ((rms[k] >> j) & 1ull) sub |= 1ull << k;
          return sub;
        };
        auto sign_word = [&](uint64_t sub) -> std::string {
          auto it = word.find(sub);
          if (it != word.end()) return it->second;
          std::string e;
          for (size_t k = 0; k < rms.size(); ++k)
            if ((sub >> k) & 1ull) e += (e.empty() ? "" : " ^ ") + sb[k];
          const std::string w = G.name("sw");
          o << "      const u32 " << w << " = " << e << ";\n";
          word[sub] = w;
          return w;
        };
        if (!table && op.t0 == 0) {
          for (int j = 0; j < J; ++j) {
            const uint64_t sub = subset(j);
            if (sub) G.set(j, "sgnw(" + G.v[j] + ", " + sign_word(sub) + ")", "");
          }
        } else if (op.t0 == 0) {  // table only: the group factor is exactly 1
          for (int j = 0; j < J; ++j) {
            const uint64_t sub = subset(j);
            const std::string t = sub ? "sgnw(" + c2(Tt[j]) + ", " + sign_word(sub) + ")" : c2(Tt[j]);
            G.set(j, "cmul(" + G.v[j] + ", " + t + ")", "");
          }
        } else {
          const std::string fv = "make_float2(" + f + "r, " + f + "i)";
          std::map<uint64_t, std::string> fs;  // term subset -> sign-adjusted group factor
          for (int j = 0; j < J; ++j) {
            const uint64_t sub = subset(j);
            std::string fj = fv;
            if (sub) {
              auto it = fs.find(sub);
              if (it == fs.end()) {
                const std::string w = sign_word(sub), n = G.name("fs");
                o << "      const float2 " << n << " = sgnw(" << fv << ", " << w << ");\n";
                it = fs.emplace(sub, n).first;
              }
              fj = it->second;
            }
            const std::string t = table ? "cmul(" + c2(Tt[j]) + ", " + fj + ")" : fj;
            G.set(j, "cmul(" + G.v[j] + ", " + t + ")", "");
          }
        }
        for (int k = 0; k < op.d0; ++k, p += 3) {
          const uint64_t rm = bits64(p[0]);
          const std::string xp = G.name("xp");
          o << "      const bool " << xp << " = " << mask_test(bits64(p[1]), G.uses_g) << ";\n";
          for (int j = 0; j < J; ++j)
            if ((rm >> j) & 1ull) G.set(j, "cmul(" + G.v[j] + ", " + c2(p[2]) + ")", xp);
        }
        break;
      }
      default:
        throw qs_error(QS_ERR_INVALID, "tile-pass specialisation: unknown device op");
    }
  }
}

// One register block as a device function of its own: the whole kernel as
// one function makes the compiler's cost grow faster than linearly with the
// number of blocks (a deep QV pass holds 30+ blocks).
std::string gen_block_fn(int b, const DevBlock& B, int T, int R, int threads, const DevOp* ops, const float2* coef,
                         bool inline_fn) {
  const uint32_t ngroups = 1u << (T - R);
  const int J = 1 << R;
  auto physh = [](uint32_t i) { return i ^ ((((i >> 4) ^ (i >> 8) ^ (i >> 12)) & 7u) << 1); };
  std::vector<uint32_t> off(J);
  for (int j = 0; j < J; ++j) {
    uint32_t x = 0;
    for (int k = 0; k < R; ++k)
      if ((j >> k) & 1) x |= 1u << B.pos[k];
    off[j] = physh(x);  // phys is linear over GF(2): phys(base|x) = phys(base)^phys(x)
  }
  Block G;
  G.v.resize(J);
  for (int j = 0; j < J; ++j) G.v[j] = "v" + std::to_string(j);
  gen_block(G, R, ops, B.op_begin, B.op_end, coef);
  std::ostringstream o;
  o << "__device__ " << (inline_fn ? "__forceinline__" : "__noinline__") << " void blk" << b << "(u64 gbase) {\n";
  o << "  float2* tile = reinterpret_cast<float2*>(smem);\n";
  if (G.uses_g) {
    o << "  const u64* dep_lo = reinterpret_cast<const u64*>(smem + " << (8 << T) << ");\n";
    o << "  const u64* dep_hi = dep_lo + 128;\n";
  }
  o << "  #pragma unroll 1\n";
  o << "  for (u32 g = threadIdx.x; g < " << ngroups << "u; g += " << threads << "u) {\n";
  o << "      u32 base = g;\n";
  for (int k = 0; k < R; ++k) o << "      base = ins0w(base, " << (int)B.pos[k] << ");\n";
  o << "      const u32 pb = phys(base);\n";
  if (G.uses_g) {
    // the interpreter evaluates global controls against 0 when the block
    // was encoded without them (pos[7] == 0)
    if (B.pos[7] != 0) o << "      const u64 gidx = gbase | dep_lo[base & 127] | dep_hi[base >> 7];\n";
    else o << "      const u64 gidx = 0ull;\n";
  }
  // Address of amplitude j: pb ^ off[j] = (pb ^ lo) + hi with lo = off[j] & 15
  // and hi = off[j] - lo, because pb is zero at the register bits (the
  // swizzle only rewrites bits 1..3).  The XOR then depends on at most 16
  // distinct lo values per group and hi becomes the load's immediate offset.
  std::map<uint32_t, std::string> lo_addr;
  auto addr = [&](int j) {
    const uint32_t lo = off[j] & 15u, hi = off[j] & ~15u;
    auto it = lo_addr.find(lo);
    if (it == lo_addr.end()) {
      const std::string n = "pa" + std::to_string(lo);
      o << "      const u32 " << n << " = pb ^ " << lo << "u;\n";
      it = lo_addr.emplace(lo, n).first;
    }
    return it->second + " + " + std::to_string(hi) + "u";
  };
  for (int j = 0; j < J; ++j) {
    const std::string a = addr(j);
    o << "      const float2 v" << j << " = tile[" << a << "];\n";
  }
  o << G.o.str();
  for (int j = 0; j < J; ++j) o << "      tile[" << addr(j) << "] = " << G.v[j] << ";\n";
  o << "  }\n}\n";
  return o.str();
}

std::string gen_pass(const DevPass& P, const DevBlock* blocks, const DevOp* ops, const float2* coef, int min_blocks) {
  const int T = P.T, R = P.R;
  const int threads = pass_threads(T, R);
  const bool inline_blocks = P.nblocks <= 4;
  std::ostringstream s;
  s << kPrelude;
  s << "extern __shared__ __align__(16) unsigned char smem[];\n";
  // dep(i) = sum_k bit_k(i) << S[k], split in two 7-bit tables (host-computed).
  s << "__device__ const u64 kDep[256] = {";
  for (int e = 0; e < 256; ++e) {
    const int part = e >> 7, x = e & 127;
    uint64_t d = 0;
    for (int k = 0; k < 7; ++k) {
      const int kk = part * 7 + k;
      if (kk < T && ((x >> k) & 1)) d |= 1ull << P.S[kk];
    }
    s << (e ? "," : "") << d << "ull";
  }
  s << "};\n";
  for (int b = 0; b < P.nblocks; ++b) s << gen_block_fn(b, blocks[b], T, R, threads, ops, coef, inline_blocks);
  s << "extern \"C\" __global__ void __launch_bounds__(" << threads << ", " << min_blocks
    << ") qs_tile_pass(float2* __restrict__ state, u64 ntiles, u32 flags, u64 nmask) {\n";
  s << "  float2* tile = reinterpret_cast<float2*>(smem);\n";
  s << "  u64* dep_lo = reinterpret_cast<u64*>(smem + " << (8 << T) << ");\n";
  s << "  const u64* dep_hi = dep_lo + 128;\n";
  s << "  for (int e = threadIdx.x; e < 256; e += " << threads << ") dep_lo[e] = kDep[e];\n";
  s << "  __syncthreads();\n";
  s << "  for (u64 t = blockIdx.x; t < ntiles; t += gridDim.x) {\n";
  s << "    u64 gbase = t;\n";
  for (int k = 0; k < T; ++k) s << "    gbase = ins0(gbase, " << P.S[k] << ");\n";
  const uint32_t npairs = 1u << (T - 1);
  s << "    if (flags & 1u) {\n"
       "      const bool first = (gbase & nmask) == 0ull;\n"
       "      for (u32 c = threadIdx.x; c < "
    << npairs << "u; c += " << threads
    << "u) {\n"
       "        const u32 i = c << 1;\n"
       "        const float x = (first && i == 0) ? 1.f : 0.f;\n"
       "        *reinterpret_cast<float4*>(tile + phys(i)) = make_float4(x, 0.f, 0.f, 0.f);\n"
       "      }\n"
       "    } else {\n"
       "      for (u32 c = threadIdx.x; c < "
    << npairs << "u; c += " << threads
    << "u) {\n"
       "        const u32 i = c << 1;\n"
       "        const u64 g = gbase | dep_lo[i & 127] | dep_hi[i >> 7];\n"
       "        const u32 d = (u32)__cvta_generic_to_shared(tile + phys(i));\n"
       "        asm volatile(\"cp.async.cg.shared.global [%0], [%1], 16;\\n\" :: \"r\"(d), \"l\"(state + g) : \"memory\");\n"
       "      }\n"
       "      asm volatile(\"cp.async.commit_group;\\ncp.async.wait_group 0;\\n\" ::: \"memory\");\n"
       "    }\n"
       "    __syncthreads();\n";
  // a from-|0> pass leaves every tile but the first of each state at +0
  s << "    if (!(flags & 1u) || (gbase & nmask) == 0ull) {\n";
  for (int b = 0; b < P.nblocks; ++b) s << "    blk" << b << "(gbase);\n    __syncthreads();\n";
  s << "    }\n";
  s << "    for (u32 c = threadIdx.x; c < " << npairs << "u; c += " << threads
    << "u) {\n"
       "      const u32 i = c << 1;\n"
       "      const u64 g = gbase | dep_lo[i & 127] | dep_hi[i >> 7];\n"
       "      *reinterpret_cast<float4*>(state + g) = *reinterpret_cast<const float4*>(tile + phys(i));\n"
       "    }\n"
       "    __syncthreads();\n"
       "  }\n"
       "}\n";
  return s.str();
}

// ------------------------------------------------ pipelined tile passes
// A persistent kernel per pass: one CTA per SM (two for 12-qubit tiles)
// walks its tiles through a ring of NS shared-memory stages.  One producer
// warp moves tiles with TMA tensor copies (cp.async.bulk.tensor): loads
// complete on the stage's "full" mbarrier, and a stage whose tile the
// consumers have finished (its "done" mbarrier) is written back by a TMA
// store and, once the store has read it, refilled with the tile NS ahead.
// The consumer warps run the pass's register blocks on the stage, so the
// next tile's load, this tile's arithmetic and the previous tile's store
// overlap.  Every wait is bounded: a wait that runs out ORs a cause into the
// handle's status word and the CTA returns after its copies in flight end.
//
// The tensor map views the state as up to 5 dimensions of 8-byte elements:
// dimension 0 covers bits [0, st1) with a box of 16 amplitudes (128 bytes,
// the 128-byte swizzle span), dimension d covers [st_d, st_{d+1}) with a box
// over the tile run that starts at st_d.  A tile's high positions form runs
// of consecutive qubits; the (at most 4) longest runs become box dimensions
// and the other positions are walked by issuing one box per combination.
// In shared memory a box is row-major over its dimensions, boxes follow one
// another, and the hardware swizzle XORs address bits [4:6] with [7:9]; so
// amplitude i of the tile (bit k = qubit S[k]) sits at a linear (XOR) image
// of i that the generator folds into every register block's addresses.
struct PipeShape {
  int rank = 0;
  int st[5] = {0, 0, 0, 0, 0};
  int boxb[5] = {0, 0, 0, 0, 0};
  int box_bits = 0;          // log2 amplitudes per box
  std::vector<int> U;        // high tile positions (global qubits) walked box by box
  std::vector<uint32_t> A;   // A[k]: shared-memory amplitude index of tile bit k (swizzled)
};

constexpr int kPipeStages = 3;

// Consumer groups: each group is a full set of compute warps (one register
// group per thread per block) and the groups take alternate tiles of the ring
// (group g: tiles g, g + groups, ...), each synchronising on a named barrier
// of its own.  Two groups put twice the warps on every scheduler, so one
// group's shared-memory phases and barrier waits overlap the other group's
// arithmetic; the price is a 120-register cap (17 warps per SM).
// QSIM_PIPE_GROUPS = 1 or 2.
int pipe_groups(int per_group) {
  static const int env = [] {
    const char* e = std::getenv("QSIM_PIPE_GROUPS");
    return e ? std::atoi(e) : 0;
  }();
  const int g = env == 1 || env == 2 ? env : 2;
  return per_group % 32 == 0 && per_group >= 64 ? g : 1;
}

bool pipe_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("QSIM_TMA_PASS");
    return !(e && std::atoi(e) == 0);
  }();
  return on;
}

// The pipelined kernel handles 10..13-qubit tiles that hold qubits 0..3
// (every tile the planner builds does) on states of at most 32 qubits (the
// dimension-0 coordinate is a signed 32-bit value).
bool pipe_shape(const DevPass& P, PipeShape& sh) {
  const int T = P.T;
  if (!pipe_enabled() || T < 10 || T > 13 || P.n_qubits > 32) return false;
  for (int k = 0; k < 4; ++k)
    if (P.S[k] != k) return false;
  std::vector<std::pair<int, int>> runs;  // (first qubit, length)
  for (int k = 4; k < T; ++k) {
    if (!runs.empty() && runs.back().first + runs.back().second == P.S[k]) ++runs.back().second;
    else runs.push_back({P.S[k], 1});
  }
  std::vector<std::pair<int, int>> pieces;  // a box dimension spans at most 256 elements
  for (auto r : runs) {
    while (r.second > 8) {
      pieces.push_back({r.first, 8});
      r.first += 8;
      r.second -= 8;
    }
    pieces.push_back(r);
  }
  std::vector<int> idx(pieces.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return pieces[a].second > pieces[b].second; });
  idx.resize(std::min<size_t>(4, idx.size()));
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return pieces[a].first < pieces[b].first; });
  sh.rank = 1 + (int)idx.size();
  sh.st[0] = 0;
  sh.boxb[0] = 4;
  sh.box_bits = 4;
  std::vector<int> smem_bit(64, -1);  // qubit -> shared-memory index bit
  for (int q = 0; q < 4; ++q) smem_bit[q] = q;
  for (size_t d = 0; d < idx.size(); ++d) {
    const auto& pc = pieces[idx[d]];
    sh.st[d + 1] = pc.first;
    sh.boxb[d + 1] = pc.second;
    for (int o = 0; o < pc.second; ++o) smem_bit[pc.first + o] = sh.box_bits + o;
    sh.box_bits += pc.second;
  }
  if (sh.rank < 2 || sh.st[1] > 31 || sh.box_bits < 7) return false;  // swizzle atoms of 1024 bytes
  int next = sh.box_bits;
  for (int k = 4; k < T; ++k)
    if (smem_bit[P.S[k]] < 0) {
      sh.U.push_back(P.S[k]);
      smem_bit[P.S[k]] = next++;
    }
  sh.A.resize(T);
  for (int k = 0; k < T; ++k) {
    const uint32_t m = 1u << smem_bit[P.S[k]];
    sh.A[k] = m ^ (((m >> 4) & 7u) << 1);  // 128-byte swizzle, in amplitude units
  }
  return true;
}

// Lane bits of a register block: the 5 non-register tile bits that put a
// warp's 32 groups on the most shared-memory banks (8-byte accesses: address
// bits 0..3; 16-byte pair accesses: bits 1..3), then the rest in order.
std::vector<int> lane_order(const std::vector<int>& nr, const std::vector<uint32_t>& A, bool pair) {
  std::vector<int> order;
  std::vector<uint32_t> basis;
  auto reduce = [&](uint32_t v) {
    for (uint32_t b : basis) v = std::min(v, v ^ b);
    return v;
  };
  for (int k : nr) {
    if (order.size() >= 5) break;
    const uint32_t v = reduce(pair ? (A[k] >> 1) & 7u : A[k] & 15u);
    if (v) {
      basis.push_back(v);
      std::sort(basis.rbegin(), basis.rend());
      order.push_back(k);
    }
  }
  for (int k : nr)
    if (std::find(order.begin(), order.end(), k) == order.end()) order.push_back(k);
  return order;
}

std::string gen_block_fn_pipe(int b, const DevBlock& B, int T, int R, int nc, const DevOp* ops, const float2* coef,
                              bool inline_fn, const std::vector<uint32_t>& A) {
  const int J = 1 << R;
  const uint32_t ngroups = 1u << (T - R);
  std::vector<int> nr;
  for (int k = 0; k < T; ++k) {
    bool reg = false;
    for (int r = 0; r < R; ++r) reg |= (B.pos[r] == k);
    if (!reg) nr.push_back(k);
  }
  const bool pair = B.pos[0] == 0;  // register bit 0 is tile bit 0: (j, j|1) are adjacent
  const std::vector<int> ord = lane_order(nr, A, pair);
  std::vector<uint32_t> off(J);
  for (int j = 0; j < J; ++j) {
    uint32_t x = 0;
    for (int k = 0; k < R; ++k)
      if ((j >> k) & 1) x ^= A[B.pos[k]];
    off[j] = x;
  }
  Block G;
  G.v.resize(J);
  for (int j = 0; j < J; ++j) G.v[j] = "v" + std::to_string(j);
  gen_block(G, R, ops, B.op_begin, B.op_end, coef);
  std::ostringstream o;
  o << "__device__ " << (inline_fn ? "__forceinline__" : "__noinline__") << " void blk" << b
    << "(u32 soff, u64 gbase, const u64* __restrict__ dep_lo, u32 tid) {\n";
  o << "  float2* tile = reinterpret_cast<float2*>(smem_raw + soff);\n";
  o << "  #pragma unroll 1\n";
  o << "  for (u32 g = tid; g < " << ngroups << "u; g += " << nc << "u) {\n";
  o << "      u32 pb = 0u;\n";
  if (G.uses_g) o << "      u32 base = 0u;\n";
  for (size_t j = 0; j < ord.size(); ++j) {
    o << "      { const u32 m_ = 0u - ((g >> " << j << ") & 1u); pb ^= m_ & " << A[ord[j]] << "u;";
    if (G.uses_g) o << " base |= m_ & " << (1u << ord[j]) << "u;";
    o << " }\n";
  }
  if (G.uses_g) {
    if (B.pos[7] != 0) o << "      const u64 gidx = gbase | dep_lo[base & 127u] | dep_lo[128u + (base >> 7)];\n";
    else o << "      const u64 gidx = 0ull;\n";
  }
  // address of amplitude j: pb ^ off[j] = (pb ^ lo) + hi (pb and hi share
  // no bit at or above bit 4, and the swizzle only rewrites bits 1..3)
  std::map<uint32_t, std::string> lo_addr;
  auto addr = [&](int j) {
    const uint32_t lo = off[j] & 15u, hi = off[j] & ~15u;
    auto it = lo_addr.find(lo);
    if (it == lo_addr.end()) {
      const std::string n = "pa" + std::to_string(lo);
      o << "      const u32 " << n << " = pb ^ " << lo << "u;\n";
      it = lo_addr.emplace(lo, n).first;
    }
    return it->second + " + " + std::to_string(hi) + "u";
  };
  for (int j = 0; j < J; ++j) {
    if (pair && (j & 1)) continue;
    const std::string a = addr(j);
    if (pair) {
      o << "      const float4 w" << j << " = *reinterpret_cast<const float4*>(tile + (" << a << "));\n";
      o << "      const float2 v" << j << " = make_float2(w" << j << ".x, w" << j << ".y);\n";
      o << "      const float2 v" << (j + 1) << " = make_float2(w" << j << ".z, w" << j << ".w);\n";
    } else {
      o << "      const float2 v" << j << " = tile[" << a << "];\n";
    }
  }
  o << G.o.str();
  for (int j = 0; j < J; ++j) {
    if (pair && (j & 1)) continue;
    if (pair)
      o << "      *reinterpret_cast<float4*>(tile + (" << addr(j) << ")) = make_float4(" << G.v[j] << ".x, " << G.v[j]
        << ".y, " << G.v[j + 1] << ".x, " << G.v[j + 1] << ".y);\n";
    else
      o << "      tile[" << addr(j) << "] = " << G.v[j] << ";\n";
  }
  o << "  }\n}\n";
  return o.str();
}

const char* kPipePrelude = R"(
struct __align__(64) TMap { unsigned long long v[16]; };
__device__ __forceinline__ u32 su32(const void* p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ u64 gtimer() { u64 t; asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t)); return t; }
__device__ __forceinline__ void mb_init(u32 b, u32 n) { asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(b), "r"(n) : "memory"); }
__device__ __forceinline__ void mb_arrive(u32 b) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" :: "r"(b) : "memory");
}
__device__ __forceinline__ void mb_expect(u32 b, u32 bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" :: "r"(b), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mb_try(u32 b, u32 par) {
  u32 ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(b), "r"(par) : "memory");
  return ok != 0u;
}
// Bounded wait for the phase of parity `par`: false once `limit` ns passed.
__device__ __forceinline__ bool mb_wait(u32 b, u32 par, u64 limit) {
  if (mb_try(b, par)) return true;
  const u64 t0 = gtimer();
  for (;;) {
    if (mb_try(b, par)) return true;
    if (gtimer() - t0 > limit) return false;
  }
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void consumers_sync(u32 grp) { asm volatile("bar.sync %0, %1;" :: "r"(grp + 1u), "n"(QS_NCG) : "memory"); }
)";

std::string gen_pass_pipe(const DevPass& P, const DevBlock* blocks, const DevOp* ops, const float2* coef,
                          const PipeShape& sh, int min_blocks) {
  const int T = P.T, R = P.R;
  const int ncg = std::min(256, 1 << (T - R));  // threads per consumer group (a multiple of 32: T - R >= 5)
  const int ngrp = pipe_groups(ncg), nc = ngrp * ncg;
  const uint32_t tile_bytes = 8u << T;
  const int nbox = 1 << sh.U.size();
  const uint32_t box_bytes = 8u << sh.box_bits;
  std::ostringstream s;
  s << kPrelude;
  s << "#define QS_NC " << nc << "\n#define QS_NCG " << ncg << "\n";
  s << kPipePrelude;
  s << "extern __shared__ __align__(1024) unsigned char smem_raw[];\n";
  s << "__device__ const u64 kDep[256] = {";
  for (int e = 0; e < 256; ++e) {
    const int part = e >> 7, x = e & 127;
    uint64_t d = 0;
    for (int k = 0; k < 7; ++k) {
      const int kk = part * 7 + k;
      if (kk < T && ((x >> k) & 1)) d |= 1ull << P.S[kk];
    }
    s << (e ? "," : "") << d << "ull";
  }
  s << "};\n";
  const bool inline_blocks = P.nblocks <= 4;
  for (int b = 0; b < P.nblocks; ++b) s << gen_block_fn_pipe(b, blocks[b], T, R, ncg, ops, coef, inline_blocks, sh.A);
  // global index of the first amplitude of tile t
  s << "__device__ __forceinline__ u64 tile_base(u64 t) {\n  u64 g = t;\n";
  for (int k = 0; k < T; ++k) s << "  g = ins0(g, " << P.S[k] << ");\n";
  s << "  return g;\n}\n";
  // one TMA box: global start g -> coordinates
  const int rk = sh.rank;
  auto coords = [&](std::ostringstream& o) {
    o << "      const int c0 = (int)(g & " << ((1ull << sh.st[1]) - 1ull) << "ull);\n";
    for (int d = 1; d < rk; ++d) {
      if (d + 1 < rk)
        o << "      const int c" << d << " = (int)((g >> " << sh.st[d] << ") & " << ((1ull << (sh.st[d + 1] - sh.st[d])) - 1ull)
          << "ull);\n";
      else
        o << "      const int c" << d << " = (int)(g >> " << sh.st[d] << ");\n";
    }
  };
  auto clist = [&]() {
    std::string c;
    for (int d = 0; d < rk; ++d) c += (d ? ", %" : "%") + std::to_string(d + 2);
    return c;
  };
  auto cargs = [&]() {
    std::string c;
    for (int d = 0; d < rk; ++d) c += ", \"r\"(c" + std::to_string(d) + ")";
    return c;
  };
  auto box_start = [&](std::ostringstream& o) {
    o << "      u64 g = gb;\n";
    for (size_t k = 0; k < sh.U.size(); ++k) o << "      if ((u >> " << k << ") & 1u) g |= " << (1ull << sh.U[k]) << "ull;\n";
  };
  s << "__device__ __forceinline__ void load_tile(const TMap* tm, u64 gb, u32 stage, u32 bar, u32 lane) {\n";
  s << "  for (u32 u = lane; u < " << nbox << "u; u += 32u) {\n";
  box_start(s);
  coords(s);
  s << "      asm volatile(\"cp.async.bulk.tensor." << rk
    << "d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {" << clist() << "}], [%" << (rk + 2)
    << "];\" :: \"r\"(stage + u * " << box_bytes << "u), \"l\"(reinterpret_cast<u64>(tm))" << cargs()
    << ", \"r\"(bar) : \"memory\");\n";
  s << "  }\n}\n";
  s << "__device__ __forceinline__ void store_tile(const TMap* tm, u64 gb, u32 stage, u32 lane) {\n";
  s << "  for (u32 u = lane; u < " << nbox << "u; u += 32u) {\n";
  box_start(s);
  coords(s);
  s << "      asm volatile(\"cp.async.bulk.tensor." << rk << "d.global.shared::cta.tile.bulk_group [%0, {"
    << [&]() {
         std::string c;
         for (int d = 0; d < rk; ++d) c += (d ? ", %" : "%") + std::to_string(d + 1);
         return c;
       }()
    << "}], [%" << (rk + 1) << "];\" :: \"l\"(reinterpret_cast<u64>(tm))" << cargs() << ", \"r\"(stage + u * "
    << box_bytes << "u) : \"memory\");\n";
  s << "  }\n  bulk_commit();\n}\n";

  const uint32_t smem_stages = kPipeStages * tile_bytes;
  s << "extern \"C\" __global__ void __launch_bounds__(" << (nc + 32) << ", " << min_blocks
    << ") qs_tile_pass(const __grid_constant__ TMap tmap, u64 ntiles, u32 flags, u64 nmask, u32* status, u64 limit) {\n";
  s << "  const u32 raw = su32(smem_raw);\n";
  s << "  const u32 pad = (1024u - (raw & 1023u)) & 1023u;\n";
  s << "  unsigned char* smem = smem_raw + pad;\n";
  s << "  const u32 stage0 = su32(smem);\n";
  s << "  u64* dep_lo = reinterpret_cast<u64*>(smem + " << smem_stages << ");\n";
  s << "  const u32 bar_full = su32(dep_lo + 256), bar_done = bar_full + " << 8 * kPipeStages << "u;\n";
  s << "  volatile u32* abort_flag = reinterpret_cast<volatile u32*>(dep_lo + 256 + " << 2 * kPipeStages << ");\n";
  s << "  const u32 tid = threadIdx.x;\n";
  s << "  for (u32 e = tid; e < 256u; e += blockDim.x) dep_lo[e] = kDep[e];\n";
  s << "  if (tid == 0) {\n";
  s << "    for (u32 k = 0; k < " << kPipeStages << "u; ++k) { mb_init(bar_full + 8u * k, 1u); mb_init(bar_done + 8u * k, "
    << ncg << "u); }\n";
  s << "    *abort_flag = 0u;\n";
  s << "    asm volatile(\"fence.mbarrier_init.release.cluster;\\nfence.proxy.async.shared::cta;\" ::: \"memory\");\n";
  s << "  }\n  __syncthreads();\n";
  s << "  const u64 mine = blockIdx.x < ntiles ? (ntiles - 1ull - blockIdx.x) / gridDim.x + 1ull : 0ull;\n";
  s << "  const bool from_zero = (flags & 1u) != 0u;\n";
  // ---- producer warp
  s << "  if (tid >= " << nc << "u) {\n";
  s << "    const u32 lane = tid & 31u;\n";
  s << "    const TMap* tm = &tmap;\n";
  s << "    bool fail = false;\n";
  s << "    long long armed[" << kPipeStages << "];\n";
  s << "    for (int k = 0; k < " << kPipeStages << "; ++k) armed[k] = -1;\n";
  s << "    u64 i = 0;\n";
  s << "    for (; i < mine; ++i) {\n";
  s << "      const u32 st = (u32)(i % " << kPipeStages << "u);\n";
  s << "      if (i >= " << kPipeStages << "u) {\n";
  s << "        const u64 j = i - " << kPipeStages << "u;\n";
  s << "        if (!mb_wait(bar_done + 8u * st, (u32)((j / " << kPipeStages << "u) & 1u), limit)) { fail = true; break; }\n";
  s << "        store_tile(tm, tile_base(blockIdx.x + j * gridDim.x), stage0 + st * " << tile_bytes << "u, lane);\n";
  s << "        bulk_wait_read0();\n";
  s << "        __syncwarp();\n";
  s << "      }\n";
  s << "      if (from_zero) { if (lane == 0u) mb_arrive(bar_full + 8u * st); }\n";
  s << "      else if (!((flags & 4u) && i == 0ull)) {\n";
  s << "        if (lane == 0u) mb_expect(bar_full + 8u * st, " << tile_bytes << "u);\n";
  s << "        __syncwarp();\n";
  s << "        load_tile(tm, tile_base(blockIdx.x + i * gridDim.x), stage0 + st * " << tile_bytes
    << "u, bar_full + 8u * st, lane);\n";
  s << "        armed[st] = (long long)i;\n";
  s << "      }\n";
  s << "    }\n";
  s << "    if (!fail) {\n";
  s << "      for (u64 j = mine > " << kPipeStages << "u ? mine - " << kPipeStages << "u : 0ull; j < mine; ++j) {\n";
  s << "        const u32 st = (u32)(j % " << kPipeStages << "u);\n";
  s << "        if (!mb_wait(bar_done + 8u * st, (u32)((j / " << kPipeStages << "u) & 1u), limit)) { fail = true; break; }\n";
  s << "        store_tile(tm, tile_base(blockIdx.x + j * gridDim.x), stage0 + st * " << tile_bytes << "u, lane);\n";
  s << "      }\n";
  s << "    }\n";
  s << "    bulk_wait0();\n";
  s << "    if (fail) {\n";
  s << "      if (lane == 0u) atomicOr(status, 1u);\n";
  s << "      // loads still in flight land in this CTA's shared memory: wait (bounded) for them\n";
  s << "      for (int k = 0; k < " << kPipeStages << "; ++k)\n";
  s << "        if (armed[k] >= 0) (void)mb_wait(bar_full + 8u * k, (u32)(((u64)armed[k] / " << kPipeStages
    << "u) & 1u), limit);\n";
  s << "    }\n";
  s << "    return;\n";
  s << "  }\n";
  // ---- consumer warps: group grp takes tiles grp, grp + ngrp, ...
  s << "  const u32 grp = tid / " << ncg << "u, lt = tid % " << ncg << "u;\n";
  // With several groups, a group reaches tile i without having consumed the
  // stage's previous tile (i - stages, another group's): the stage's "full"
  // phase for that tile may still be open, and a parity wait would see the
  // phase before it (same parity) as complete.  So the group first waits for
  // the "done" phase of tile i - stages (its own arrivals completed the one
  // before), which also means that tile's "full" phase is over; then the
  // "full" wait for tile i is unambiguous.
  s << "  for (u64 i = grp; i < mine; i += " << ngrp << "u) {\n";
  s << "    const u32 st = (u32)(i % " << kPipeStages << "u);\n";
  s << "    bool ok = true;\n";
  if (ngrp > 1)
    s << "    if (i >= " << kPipeStages << "u) ok = mb_wait(bar_done + 8u * st, (u32)(((i - " << kPipeStages << "u) / "
      << kPipeStages << "u) & 1u), limit);\n";
  s << "    if (!ok || !mb_wait(bar_full + 8u * st, (u32)((i / " << kPipeStages << "u) & 1u), limit)) *abort_flag = 1u;\n";
  s << "    consumers_sync(grp);\n";
  s << "    if (*abort_flag) { if (lt == 0u) atomicOr(status, 2u); return; }\n";
  s << "    const u32 soff = pad + st * " << tile_bytes << "u;\n";
  s << "    float2* tile = reinterpret_cast<float2*>(smem_raw + soff);\n";
  s << "    const u64 gbase = tile_base(blockIdx.x + i * gridDim.x);\n";
  s << "    if (from_zero) {\n";
  s << "      float4* t4 = reinterpret_cast<float4*>(tile);\n";
  s << "      for (u32 c = lt; c < " << (tile_bytes / 16) << "u; c += " << ncg
    << "u) t4[c] = make_float4(0.f, 0.f, 0.f, 0.f);\n";
  s << "      if (lt == 0u && (gbase & nmask) == 0ull) tile[0] = make_float2(1.f, 0.f);  // lt 0 zeroed t4[0]\n";
  s << "      consumers_sync(grp);\n";
  s << "    }\n";
  // a from-|0> pass leaves every tile but the first of each state at +0
  // (the interpreter skips them too, so both give the same bits)
  s << "    if (!from_zero || (gbase & nmask) == 0ull) {\n";
  for (int b = 0; b < P.nblocks; ++b) {
    s << "    blk" << b << "(soff, gbase, dep_lo, lt);\n";
    if (b + 1 < P.nblocks) s << "    consumers_sync(grp);\n";
  }
  s << "    }\n";
  s << "    asm volatile(\"fence.proxy.async.shared::cta;\" ::: \"memory\");\n";
  s << "    mb_arrive(bar_done + 8u * st);\n";
  s << "  }\n";
  s << "}\n";
  return s.str();
}

int pipe_smem(int T) { return kPipeStages * (8 << T) + 1024 + 256 * 8 + 2 * kPipeStages * 8 + 16; }
int pipe_threads(int T, int R) {
  const int per_group = std::min(256, 1 << (T - R));
  return pipe_groups(per_group) * per_group + 32;
}

uint64_t fnv1a(const std::string& s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char ch : s) {
    h ^= ch;
    h *= 1099511628211ull;
  }
  return h;
}

// Compiled passes, per device, keyed by a hash of their source (plans of the
// same circuit share kernels; modules live until the process exits).  Heap
// objects that are never destroyed: a background compile may still be running
// while static destructors run at exit.
struct Cache {
  std::mutex mu;
  std::unordered_map<uint64_t, std::pair<std::string, JitPass>> map[64];
};
Cache& cache() {
  static Cache* c = new Cache;
  return *c;
}

bool nvrtc_compile(const std::string& src, std::string& cubin, std::string& err) {
  nvrtcProgram prog = nullptr;
  if (g_api.CreateProgram(&prog, src.c_str(), "qs_tile_pass.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
    err = "nvrtcCreateProgram failed";
    return false;
  }
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=true", "-default-device"};
  const nvrtcResult rc = g_api.CompileProgram(prog, 4, opts);
  if (rc != NVRTC_SUCCESS) {
    size_t n = 0;
    g_api.GetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    if (n) g_api.GetProgramLog(prog, &log[0]);
    err = "NVRTC: " + log.substr(0, 600);
    g_api.DestroyProgram(&prog);
    return false;
  }
  size_t nb = 0;
  g_api.GetCUBINSize(prog, &nb);
  cubin.assign(nb, '\0');
  g_api.GetCUBIN(prog, &cubin[0]);
  g_api.DestroyProgram(&prog);
  return true;
}

// Register-allocation hint: the CTAs per SM that the tile's shared memory
// allows (228 KiB per SM, 1 KiB reserved per CTA), capped so that a thread
// keeps at least 128 registers.
int min_blocks_for(int smem, int threads, int R) {
  const int by_smem = (228 * 1024) / (smem + 1024);
  const int by_regs = 65536 / (threads * (R >= 6 ? 192 : 128));
  return std::max(1, std::min(std::min(4, by_smem), by_regs));
}

}  // namespace

int qs_jit_env_mode() {
  const char* e = std::getenv("QSIM_JIT");
  if (!e || !*e) return 1;
  return std::max(0, std::min(2, std::atoi(e)));
}

bool qs_jit_available(std::string* why) {
  std::call_once(g_api_once, load_api);
  if (why) *why = !g_api.nvrtc_ok ? g_api.why_nvrtc : g_api.why_driver;
  return g_api.nvrtc_ok && g_api.driver_ok;
}

// Host-only check: generates and compiles (without loading) every pass.
bool qs_jit_compile_only(const qs_plan_s* p, std::string& err) {
  std::call_once(g_api_once, load_api);
  if (!g_api.nvrtc_ok) {
    err = g_api.why_nvrtc;
    return false;
  }
  const char* dump = std::getenv("QSIM_JIT_DUMP");  // directory for the generated sources
  for (size_t i = 0; i < p->pass_offsets.size(); ++i) {
    const std::string src = qs_jit_source(p, i);
    if (dump && *dump) {
      const std::string fn = std::string(dump) + "/pass" + std::to_string(i) + ".cu";
      if (FILE* f = std::fopen(fn.c_str(), "w")) {
        std::fwrite(src.data(), 1, src.size(), f);
        std::fclose(f);
      }
    }
    std::string cubin;
    if (!nvrtc_compile(src, cubin, err)) return false;
  }
  return true;
}

// Source of one pass from its device-program bytes (header first).
static std::string pass_source(const char* base) {
  const DevPass& P = *reinterpret_cast<const DevPass*>(base);
  const DevBlock* blocks = reinterpret_cast<const DevBlock*>(base + P.block_off);
  const DevOp* ops = reinterpret_cast<const DevOp*>(base + P.op_off);
  const float2* coef = reinterpret_cast<const float2*>(base + P.coef_off);
  PipeShape sh;
  if (P.R <= 5 && pipe_shape(P, sh))
    return gen_pass_pipe(P, blocks, ops, coef, sh, min_blocks_for(pipe_smem(P.T), pipe_threads(P.T, P.R), P.R));
  return gen_pass(P, blocks, ops, coef, min_blocks_for(pass_smem(P.T), pass_threads(P.T, P.R), P.R));
}

// Launch shape of a pass's kernel (pipelined or single-buffered).
static void pass_launch_shape(const char* base, JitPass& K) {
  const DevPass& P = *reinterpret_cast<const DevPass*>(base);
  PipeShape sh;
  if (P.R <= 5 && pipe_shape(P, sh)) {
    K.pipe = 1;
    K.threads = pipe_threads(P.T, P.R);
    K.smem = pipe_smem(P.T);
    K.rank = sh.rank;
    for (int d = 0; d < 5; ++d) {
      K.st[d] = sh.st[d];
      K.boxb[d] = sh.boxb[d];
    }
  } else {
    K.pipe = 0;
    K.threads = pass_threads(P.T, P.R);
    K.smem = pass_smem(P.T);
  }
}

std::string qs_jit_source(const qs_plan_s* p, size_t i) { return pass_source(p->blob.data() + p->pass_offsets[i]); }

// A specialisation job: the plan's pass sources, the kernels found in the
// cache and the ones still to compile.  Shared by the plan and, for tiered
// compilation, the background thread that compiles it.
struct JitJob {
  int device = 0;
  std::vector<std::string> srcs;   // generated sources (passes to compile only)
  std::vector<std::string> progs;  // cache keys: program bytes + generator knobs
  std::vector<uint64_t> keys;
  std::vector<int> T, R;
  std::vector<JitPass> out;
  std::vector<size_t> todo;  // passes not in the cache
  std::string err;
  std::atomic<int> state{0};  // 0 pending, 1 ready, 2 failed
};

namespace {

// Cache key of a pass: its device-program bytes (header, blocks, ops,
// coefficients) plus the generator's tuning knobs; the source is generated
// only for passes not in the cache.
std::string pass_key(const qs_plan_s* p, size_t i) {
  const char* base = p->blob.data() + p->pass_offsets[i];
  const DevPass& P = *reinterpret_cast<const DevPass*>(base);
  std::string k(base, base + P.bytes);
  k += "|t" + std::to_string(pass_threads(P.T, P.R)) + "|s" + std::to_string(scalar_every()) + "|p" +
       std::to_string(pipe_enabled() ? 1 : 0) + "|g" + std::to_string(pipe_groups(256));
  return k;
}

std::shared_ptr<JitJob> make_job(const qs_plan_s* p, int device) {
  auto J = std::make_shared<JitJob>();
  J->device = device;
  const size_t np = p->pass_offsets.size();
  J->srcs.resize(np);
  J->progs.resize(np);
  J->keys.resize(np);
  J->out.resize(np);
  for (size_t i = 0; i < np; ++i) {
    const DevPass& P = *reinterpret_cast<const DevPass*>(p->blob.data() + p->pass_offsets[i]);
    J->T.push_back(P.T);
    J->R.push_back(P.R);
    J->progs[i] = pass_key(p, i);
    J->keys[i] = fnv1a(J->progs[i]);
  }
  {
    Cache& C = cache();
    std::lock_guard<std::mutex> lk(C.mu);
    for (size_t i = 0; i < np; ++i) {
      auto it = C.map[device].find(J->keys[i]);
      if (it != C.map[device].end() && it->second.first == J->progs[i]) J->out[i] = it->second.second;
      else J->todo.push_back(i);
    }
  }
  // sources are generated by run_job, from the program bytes held in progs
  if (J->todo.empty()) J->state = 1;
  return J;
}

// Compiles the missing passes on up to `max_threads` host threads, then loads
// them (on this thread, with the device's primary context current).
void run_job(JitJob& J, unsigned max_threads) {
  const size_t nt_all = J.todo.size();
  for (size_t i : J.todo)
    if (J.srcs[i].empty()) J.srcs[i] = pass_source(J.progs[i].data());
  std::vector<std::string> cubins(J.srcs.size()), errs(J.srcs.size());
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nt = std::max(1u, std::min<unsigned>(std::min(max_threads, hw), (unsigned)nt_all));
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; ++t)
    pool.emplace_back([&, t]() {
      for (size_t k = t; k < nt_all; k += nt) {
        const size_t i = J.todo[k];
        if (!nvrtc_compile(J.srcs[i], cubins[i], errs[i]) && errs[i].empty()) errs[i] = "compile failed";
      }
    });
  for (auto& th : pool) th.join();
  for (size_t i : J.todo)
    if (cubins[i].empty()) {
      J.err = errs[i];
      J.state = 2;
      return;
    }
  if (cudaSetDevice(J.device) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
    J.err = "cannot make the device current for module loading";
    J.state = 2;
    return;
  }
  Cache& C = cache();
  for (size_t i : J.todo) {
    CUmodule mod = nullptr;
    CUfunction fn = nullptr;
    if (g_api.ModuleLoadData(&mod, cubins[i].data()) != CUDA_SUCCESS ||
        g_api.ModuleGetFunction(&fn, mod, "qs_tile_pass") != CUDA_SUCCESS) {
      J.err = "loading a specialised tile pass failed";
      J.state = 2;
      return;
    }
    JitPass K;
    K.fn = fn;
    pass_launch_shape(J.progs[i].data(), K);
    if (K.pipe && !g_api.EncodeTiled) {
      J.err = "cuTensorMapEncodeTiled is missing from the driver";
      J.state = 2;
      return;
    }
    if (g_api.FuncSetAttribute(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, K.smem) != CUDA_SUCCESS ||
        g_api.Occupancy(&K.per_sm, fn, K.threads, (size_t)K.smem) != CUDA_SUCCESS || K.per_sm < 1) {
      J.err = "a specialised tile pass does not fit on an SM";
      J.state = 2;
      return;
    }
    J.out[i] = K;
    std::lock_guard<std::mutex> lk(C.mu);
    C.map[J.device][J.keys[i]] = {J.progs[i], K};
  }
  J.state = 1;
}

// One background thread compiles queued jobs in arrival order (each with up
// to 8 NVRTC threads), so that many large plans in flight never start more
// compiles than that.  Jobs whose plan has been destroyed are skipped.  At
// exit the thread finishes the job in hand and stops.
struct Background {
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::weak_ptr<JitJob>> queue;
  std::thread worker;
  bool stop = false;
};
Background& background() {
  static Background* b = new Background;
  return *b;
}
void background_loop() {
  Background& B = background();
  for (;;) {
    std::shared_ptr<JitJob> J;
    {
      std::unique_lock<std::mutex> lk(B.mu);
      B.cv.wait(lk, [&] { return B.stop || !B.queue.empty(); });
      if (B.stop) return;
      J = B.queue.front().lock();
      B.queue.pop_front();
    }
    if (J && J->state.load() == 0) run_job(*J, 8);
  }
}
void stop_background() {
  Background& B = background();
  {
    std::lock_guard<std::mutex> lk(B.mu);
    B.stop = true;
  }
  B.cv.notify_all();
  if (B.worker.joinable()) B.worker.join();
}
void enqueue(const std::shared_ptr<JitJob>& J) {
  Background& B = background();
  std::lock_guard<std::mutex> lk(B.mu);
  if (B.stop) return;
  if (!B.worker.joinable()) {
    B.worker = std::thread(background_loop);
    std::atexit(stop_background);
  }
  B.queue.push_back(J);
  B.cv.notify_one();
}

}  // namespace

// Synchronous specialisation: every pass compiled (or found in the cache)
// before returning.  On failure the plan keeps running on the generic kernel
// and `err` says why.
bool qs_jit_compile_plan(qs_context* h, qs_plan_s* p, std::string& err) {
  if (!qs_jit_available(&err)) return false;
  QS_CHECK_ARG(h->device >= 0 && h->device < 64, "device index out of range");
  auto J = make_job(p, h->device);
  if (J->state == 0) run_job(*J, 16);
  if (J->state != 1) {
    err = J->err;
    return false;
  }
  p->jit = J->out;
  return true;
}

// Tiered specialisation.  First execution: the pass sources are generated and
// looked up in the kernel cache; a full hit specialises the plan at once.
// Second execution (the plan is being reused): the missing passes are queued
// for the background compiler.  Later executions switch over once it is done.
void qs_jit_tiered(qs_context* h, qs_plan_s* p) {
  if (!p->jit.empty()) return;
  if (!p->jit_tried) {
    p->jit_tried = true;
    std::string why;
    if (!qs_jit_available(&why)) {
      p->jit_err = why;
      return;
    }
    QS_CHECK_ARG(h->device >= 0 && h->device < 64, "device index out of range");
    auto J = make_job(p, h->device);
    if (J->state == 1) p->jit = J->out;
    else p->jit_job = J;
    return;
  }
  if (!p->jit_job) return;
  if (!p->jit_queued) {
    p->jit_queued = true;
    enqueue(p->jit_job);
    return;
  }
  const int st = p->jit_job->state.load();
  if (st == 1) p->jit = p->jit_job->out;
  if (st == 2) p->jit_err = p->jit_job->err;
  if (st != 0) p->jit_job.reset();
}

// Tensor map of `state` (n_states states of n qubits back to back) for a
// pipelined pass: dimension d starts at qubit st[d] and ends where the next
// starts (the last one spans the rest of the buffer); 8-byte elements, a box
// of 16 elements x 2^boxb[d], 128-byte swizzle.
static void encode_state_map(const JitPass& K, void* state, uint64_t total_amps, CUtensorMap* m) {
  cuuint64_t dim[5], stride[4];
  cuuint32_t box[5], estr[5];
  const int rk = K.rank;
  for (int d = 0; d < rk; ++d) {
    const int lo = K.st[d];
    dim[d] = d + 1 < rk ? (1ull << (K.st[d + 1] - lo)) : (total_amps >> lo);
    box[d] = 1u << K.boxb[d];
    estr[d] = 1;
    if (d > 0) stride[d - 1] = (1ull << lo) * 8ull;
  }
  const CUresult rc = g_api.EncodeTiled(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rk, state, dim, stride, box, estr,
                                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS)
    throw qs_error(QS_ERR_CUDA, "cuTensorMapEncodeTiled failed for a pipelined tile pass (CUresult " +
                                    std::to_string((int)rc) + ")");
}

void qs_jit_launch(qs_context* h, const qs_plan_s* p, size_t i, void* state, uint64_t ntiles, uint32_t flags) {
  const JitPass& K = p->jit[i];
  float2* st = static_cast<float2*>(state);
  uint64_t nt = ntiles;
  uint32_t fl = flags;
  uint64_t nmask = (1ull << p->n_qubits) - 1ull;
  const uint64_t grid = std::min<uint64_t>(ntiles, (uint64_t)h->sm_count * (uint64_t)K.per_sm);
  if (grid == 0) return;
  CUresult rc;
  if (K.pipe) {
    alignas(64) CUtensorMap tm;
    const int T = p->pass_T[i];
    encode_state_map(K, state, ntiles << T, &tm);
    // bounded waits: 4 s (a tile's copy takes microseconds; the margin covers
    // time slicing with other processes); the wait test uses 50 ms
    uint64_t limit = 4000000000ull;
    if (h->wait_test == 1) {
      fl |= 4u;
      limit = 50000000ull;
      h->wait_test = 0;
    }
    uint32_t* status = h->dev_status;
    void* args[] = {&tm, &nt, &fl, &nmask, &status, &limit};
    rc = g_api.LaunchKernel((CUfunction)K.fn, (unsigned)grid, 1, 1, (unsigned)K.threads, 1, 1, (unsigned)K.smem,
                            (CUstream)h->stream, args, nullptr);
  } else {
    void* args[] = {&st, &nt, &fl, &nmask};
    rc = g_api.LaunchKernel((CUfunction)K.fn, (unsigned)grid, 1, 1, (unsigned)K.threads, 1, 1, (unsigned)K.smem,
                            (CUstream)h->stream, args, nullptr);
  }
  if (rc != CUDA_SUCCESS)
    throw qs_error(QS_ERR_CUDA, "launch of a specialised tile pass failed (CUresult " + std::to_string((int)rc) + ")");
  qs_after_launch(h, "qs_tile_pass");
}
