// qs_pass.cu — the fused tile-pass kernel.
//
// One launch applies one pass of a host-built plan (qs_plan.cpp) to one or
// more states.  A pass is defined by a tile: T qubit positions S[0..T-1]
// (always including the low qubits, so that a tile is a set of contiguous
// runs of amplitudes in HBM).  Each CTA loops over tiles:
//
//   1. HBM -> shared memory with 16-byte cp.async (swizzled layout),
//   2. for each register block (R <= 5 tile positions): every thread gathers
//      the 2^R amplitudes of its group into registers, runs the block's ops
//      there (dense 1Q/2Q, exact X/SWAP/Y/negation, phases and diagonals,
//      with controls on any qubit), and scatters them back,
//   3. shared memory -> HBM with 16-byte stores, in place.
//
// The state is therefore read and written once per pass however many gates
// the pass holds.  Gate qubit positions are compile-time template arguments
// (dispatched by a switch), so the amplitudes stay in registers.
#include "qs_api.h"
#include "qs_common.cuh"
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <set>
#include <tuple>

using namespace qs;

namespace {

// Shared-memory swizzle: XOR bits 1..3 of the index with a fold of the higher
// bits.  It is linear over GF(2) (phys(a^b) = phys(a)^phys(b)), keeps the
// 16-byte pairs (2k, 2k+1) together, and spreads lanes that differ only in
// high tile bits over different banks.
__device__ __forceinline__ uint32_t phys(uint32_t i) {
  return i ^ ((((i >> 4) ^ (i >> 8) ^ (i >> 12)) & 7u) << 1);
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}
// Largest dynamic shared memory a pass launch may ask for: a 2^14-amplitude
// tile (128 KiB) + coefficient pool + dep tables.
constexpr int kMaxPassSmem = 200 * 1024;

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// ----------------------------------------------------- register ops -------
// v[j] holds amplitude j of the thread's group (bit k of j = register
// position k).  "gp" is the controls-read-from-the-global-index predicate,
// "rc" the mask of controls among the register bits.

// single-rounding complex product (FMA form)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -__fmul_rn(a.y, b.y)), fmaf(a.x, b.y, __fmul_rn(a.y, b.x)));
}

template <int R, int A>
__device__ __forceinline__ void op_u1(float2 (&v)[1 << R], const float2* __restrict__ c, unsigned rc, bool gp) {
  if constexpr (A < R) {
    const float2 g00 = c[0], g01 = c[1], g10 = c[2], g11 = c[3];
    if (rc == 0 && gp) {
#pragma unroll
      for (int j = 0; j < (1 << R); ++j) {
        if (j & (1 << A)) continue;
        const int k = j | (1 << A);
        const float2 a0 = v[j], a1 = v[k];
        v[j] = cfma2(g00, a0, g01, a1);
        v[k] = cfma2(g10, a0, g11, a1);
      }
      return;
    }
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & (1 << A)) continue;
      const int k = j | (1 << A);
      const bool p = gp && ((j & rc) == rc);
      float2 a0 = v[j], a1 = v[k];
      float2 n0 = cfma2(g00, a0, g01, a1);
      float2 n1 = cfma2(g10, a0, g11, a1);
      v[j] = p ? n0 : a0;
      v[k] = p ? n1 : a1;
    }
  }
}

// Real rotation [[c, -s], [s, c]]: 4 FP32 instructions per amplitude.
template <int R, int A>
__device__ __forceinline__ void op_ry(float2 (&v)[1 << R], float2 cs, unsigned rc, bool gp) {
  if constexpr (A < R) {
    const float co = cs.x, si = cs.y;
    if (rc == 0 && gp) {
#pragma unroll
      for (int j = 0; j < (1 << R); ++j) {
        if (j & (1 << A)) continue;
        const int k = j | (1 << A);
        const float2 a0 = v[j], a1 = v[k];
        v[j] = make_float2(fmaf(co, a0.x, -__fmul_rn(si, a1.x)), fmaf(co, a0.y, -__fmul_rn(si, a1.y)));
        v[k] = make_float2(fmaf(si, a0.x, __fmul_rn(co, a1.x)), fmaf(si, a0.y, __fmul_rn(co, a1.y)));
      }
      return;
    }
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & (1 << A)) continue;
      const int k = j | (1 << A);
      const bool p = gp && ((j & rc) == rc);
      const float2 a0 = v[j], a1 = v[k];
      const float2 n0 = make_float2(fmaf(co, a0.x, -__fmul_rn(si, a1.x)), fmaf(co, a0.y, -__fmul_rn(si, a1.y)));
      const float2 n1 = make_float2(fmaf(si, a0.x, __fmul_rn(co, a1.x)), fmaf(si, a0.y, __fmul_rn(co, a1.y)));
      v[j] = p ? n0 : a0;
      v[k] = p ? n1 : a1;
    }
  }
}

// Uncontrolled dense 4x4 (DK_U2): no predication.
template <int R, int A, int B>
__device__ __forceinline__ void op_u2(float2 (&v)[1 << R], const float2* __restrict__ c) {
  if constexpr (A < B && B < R) {
    float2 g[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) g[i] = c[i];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & ((1 << A) | (1 << B))) continue;
      const int j1 = j | (1 << A), j2 = j | (1 << B), j3 = j1 | (1 << B);
      const float2 a0 = v[j], a1 = v[j1], a2 = v[j2], a3 = v[j3];
      v[j] = cfma4(g + 0, a0, a1, a2, a3);
      v[j1] = cfma4(g + 4, a0, a1, a2, a3);
      v[j2] = cfma4(g + 8, a0, a1, a2, a3);
      v[j3] = cfma4(g + 12, a0, a1, a2, a3);
    }
  }
}

// Controlled dense 4x4 (DK_CU2): each quad is updated where its controls hold.
template <int R, int A, int B>
__device__ __forceinline__ void op_cu2(float2 (&v)[1 << R], const float2* __restrict__ c, unsigned rc, bool gp) {
  if constexpr (A < B && B < R) {
    float2 g[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) g[i] = c[i];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & ((1 << A) | (1 << B))) continue;
      const int j1 = j | (1 << A), j2 = j | (1 << B), j3 = j1 | (1 << B);
      const float2 a0 = v[j], a1 = v[j1], a2 = v[j2], a3 = v[j3];
      const float2 n0 = cfma4(g + 0, a0, a1, a2, a3);
      const float2 n1 = cfma4(g + 4, a0, a1, a2, a3);
      const float2 n2 = cfma4(g + 8, a0, a1, a2, a3);
      const float2 n3 = cfma4(g + 12, a0, a1, a2, a3);
      const bool p = gp && ((j & rc) == rc);
      v[j] = p ? n0 : a0;
      v[j1] = p ? n1 : a1;
      v[j2] = p ? n2 : a2;
      v[j3] = p ? n3 : a3;
    }
  }
}

template <int R, int A>
__device__ __forceinline__ void op_x(float2 (&v)[1 << R], unsigned rc, bool gp) {
  if constexpr (A < R) {
    if (rc == 0 && gp) {
#pragma unroll
      for (int j = 0; j < (1 << R); ++j) {
        if (j & (1 << A)) continue;
        const float2 t = v[j];
        v[j] = v[j | (1 << A)];
        v[j | (1 << A)] = t;
      }
      return;
    }
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & (1 << A)) continue;
      const int k = j | (1 << A);
      const bool p = gp && ((j & rc) == rc);
      float2 a0 = v[j], a1 = v[k];
      v[j] = p ? a1 : a0;
      v[k] = p ? a0 : a1;
    }
  }
}

template <int R, int A>
__device__ __forceinline__ void op_y(float2 (&v)[1 << R], unsigned rc, bool gp) {
  if constexpr (A < R) {
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & (1 << A)) continue;
      const int k = j | (1 << A);
      const bool p = gp && ((j & rc) == rc);
      float2 a0 = v[j], a1 = v[k];
      // Y|0> = i|1>, Y|1> = -i|0>:  new0 = -i*a1, new1 = i*a0
      float2 n0 = make_float2(a1.y, -a1.x);
      float2 n1 = make_float2(-a0.y, a0.x);
      v[j] = p ? n0 : a0;
      v[k] = p ? n1 : a1;
    }
  }
}

template <int R, int A, int B>
__device__ __forceinline__ void op_swap(float2 (&v)[1 << R], unsigned rc, bool gp) {
  if constexpr (A < B && B < R) {
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & ((1 << A) | (1 << B))) continue;
      const int ja = j | (1 << A), jb = j | (1 << B);
      const bool p = gp && ((j & rc) == rc);
      float2 a = v[ja], b = v[jb];
      v[ja] = p ? b : a;
      v[jb] = p ? a : b;
    }
  }
}

// Kronecker layer: a scaled rotation on every register bit set in `mask`
// (c[k] = (t, form), see DK_KRY), fully unrolled at compile-time positions;
// one dispatch for up to R gates, one FMA per output component.
template <int R, int K>
__device__ __forceinline__ void kry_stage(float2 (&v)[1 << R], float2 tf) {
  // packed FP32x2 FMAs; each lane is the scalar fmaf of the same operands
  const float2 tt = make_float2(tf.x, tf.x), nt = make_float2(-tf.x, -tf.x);
  if (tf.y == 0.f) {
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & (1 << K)) continue;
      const int k = j | (1 << K);
      const float2 a0 = v[j], a1 = v[k];
      v[j] = __ffma2_rn(nt, a1, a0);
      v[k] = __ffma2_rn(tt, a0, a1);
    }
  } else {
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & (1 << K)) continue;
      const int k = j | (1 << K);
      const float2 a0 = v[j], a1 = v[k];
      v[j] = make_float2(fmaf(tt.x, a0.x, -a1.x), fmaf(tt.x, a0.y, -a1.y));  // negated addend: scalar FMAs
      v[k] = __ffma2_rn(tt, a1, a0);
    }
  }
}

template <int R, int K>
__device__ __forceinline__ void ku1_stage(float2 (&v)[1 << R], const float2* __restrict__ c) {
  const float2 g00 = c[0], g01 = c[1], g10 = c[2], g11 = c[3];
#pragma unroll
  for (int j = 0; j < (1 << R); ++j) {
    if (j & (1 << K)) continue;
    const int k = j | (1 << K);
    const float2 a0 = v[j], a1 = v[k];
    v[j] = cfma2(g00, a0, g01, a1);
    v[k] = cfma2(g10, a0, g11, a1);
  }
}

template <int R>
__device__ __forceinline__ void op_kry(float2 (&v)[1 << R], const float2* __restrict__ c, unsigned mask) {
  if constexpr (R > 0) if (mask & 1u) kry_stage<R, 0>(v, c[0]);
  if constexpr (R > 1) if (mask & 2u) kry_stage<R, 1>(v, c[1]);
  if constexpr (R > 2) if (mask & 4u) kry_stage<R, 2>(v, c[2]);
  if constexpr (R > 3) if (mask & 8u) kry_stage<R, 3>(v, c[3]);
  if constexpr (R > 4) if (mask & 16u) kry_stage<R, 4>(v, c[4]);
}

// Parity rotation (DK_XRY) on register bits A < B: pairs j (bit A clear) and
// j ^ (A|B), with the even-parity (bit B clear) or odd-parity coefficients.
template <int R, int A, int B>
__device__ __forceinline__ void op_xry(float2 (&v)[1 << R], const float2* __restrict__ c) {
  if constexpr (A < B && B < R) {
    const float2 ce = c[0], co = c[1];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & (1 << A)) continue;
      const int k = j ^ ((1 << A) | (1 << B));
      const float2 tf = (j & (1 << B)) ? co : ce;
      const float2 tt = make_float2(tf.x, tf.x), nt = make_float2(-tf.x, -tf.x);
      const float2 a0 = v[j], a1 = v[k];
      if (tf.y == 0.f) {
        v[j] = __ffma2_rn(nt, a1, a0);
        v[k] = __ffma2_rn(tt, a0, a1);
      } else {
        v[j] = make_float2(fmaf(tt.x, a0.x, -a1.x), fmaf(tt.x, a0.y, -a1.y));
        v[k] = __ffma2_rn(tt, a1, a0);
      }
    }
  }
}

template <int R>
__device__ __forceinline__ void op_scale(float2 (&v)[1 << R], float f) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j) v[j] = make_float2(__fmul_rn(v[j].x, f), __fmul_rn(v[j].y, f));
}

template <int R>
__device__ __forceinline__ void op_ku1(float2 (&v)[1 << R], const float2* __restrict__ c, unsigned mask) {
  if constexpr (R > 0) if (mask & 1u) ku1_stage<R, 0>(v, c + 0);
  if constexpr (R > 1) if (mask & 2u) ku1_stage<R, 1>(v, c + 4);
  if constexpr (R > 2) if (mask & 4u) ku1_stage<R, 2>(v, c + 8);
  if constexpr (R > 3) if (mask & 8u) ku1_stage<R, 3>(v, c + 12);
  if constexpr (R > 4) if (mask & 16u) ku1_stage<R, 4>(v, c + 16);
}

__device__ __forceinline__ uint64_t bits64(float2 f) {
  return (uint64_t)__float_as_uint(f.x) | ((uint64_t)__float_as_uint(f.y) << 32);
}

// Merged diagonal (layout written by encode_dtab in qs_plan.cpp).
template <int R>
__device__ __forceinline__ void op_dtab(float2 (&v)[1 << R], const DevOp& op, const float2* __restrict__ c,
                                        uint64_t gidx) {
  const float2* p = c;
  const bool table = op.rc & 1;
  const float2* T = p;
  if (table) p += (1 << R);
  float fr = 1.f, fi = 0.f;
  for (int k = 0; k < op.t0; ++k) {
    const uint64_t gm = bits64(p[0]);
    const float2 w = p[1];
    p += 2;
    if ((gidx & gm) == gm) {
      const float r = fmaf(fr, w.x, -__fmul_rn(fi, w.y));
      fi = fmaf(fr, w.y, __fmul_rn(fi, w.x));
      fr = r;
    }
  }
  uint32_t m = 0;
  for (int k = 0; k < op.t1; ++k) {
    const uint32_t rm = __float_as_uint(p[0].x);
    const uint64_t gm = bits64(p[1]);
    p += 2;
    if ((gidx & gm) == gm) m ^= rm;
  }
  const float2 f = make_float2(fr, fi);
  if (!table && op.t0 == 0) {  // signs only (CZ runs): flip sign bits
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      const uint32_t sb = (m << (31 - j)) & 0x80000000u;
      v[j].x = __uint_as_float(__float_as_uint(v[j].x) ^ sb);
      v[j].y = __uint_as_float(__float_as_uint(v[j].y) ^ sb);
    }
  } else if (op.t0 == 0) {  // table only: the group factor is exactly 1
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      const uint32_t sb = (m << (31 - j)) & 0x80000000u;
      const float2 t = make_float2(__uint_as_float(__float_as_uint(T[j].x) ^ sb),
                                   __uint_as_float(__float_as_uint(T[j].y) ^ sb));
      v[j] = cmul(v[j], t);
    }
  } else {  // the sign goes onto the group factor, before the table product
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      const uint32_t sb = (m << (31 - j)) & 0x80000000u;
      const float2 fs = make_float2(__uint_as_float(__float_as_uint(f.x) ^ sb), __uint_as_float(__float_as_uint(f.y) ^ sb));
      v[j] = cmul(v[j], table ? cmul(T[j], fs) : fs);
    }
  }
  for (int k = 0; k < op.d0; ++k) {
    const uint32_t rm = __float_as_uint(p[0].x);
    const uint64_t gm = bits64(p[1]);
    const float2 w = p[2];
    p += 3;
    if ((gidx & gm) == gm) {
#pragma unroll
      for (int j = 0; j < (1 << R); ++j)
        if ((rm >> j) & 1u) v[j] = cmul(v[j], w);
    }
  }
}

#define CASES_1(F, ...)                                                          \
  case 0: F<R, 0>(__VA_ARGS__); break;                                           \
  case 1: F<R, 1>(__VA_ARGS__); break;                                           \
  case 2: F<R, 2>(__VA_ARGS__); break;                                           \
  case 3: F<R, 3>(__VA_ARGS__); break;                                           \
  case 4: F<R, 4>(__VA_ARGS__); break;

#define CASES_2(F, ...)                                                          \
  case 0 * 8 + 1: F<R, 0, 1>(__VA_ARGS__); break;                                \
  case 0 * 8 + 2: F<R, 0, 2>(__VA_ARGS__); break;                                \
  case 0 * 8 + 3: F<R, 0, 3>(__VA_ARGS__); break;                                \
  case 0 * 8 + 4: F<R, 0, 4>(__VA_ARGS__); break;                                \
  case 1 * 8 + 2: F<R, 1, 2>(__VA_ARGS__); break;                                \
  case 1 * 8 + 3: F<R, 1, 3>(__VA_ARGS__); break;                                \
  case 1 * 8 + 4: F<R, 1, 4>(__VA_ARGS__); break;                                \
  case 2 * 8 + 3: F<R, 2, 3>(__VA_ARGS__); break;                                \
  case 2 * 8 + 4: F<R, 2, 4>(__VA_ARGS__); break;                                \
  case 3 * 8 + 4: F<R, 3, 4>(__VA_ARGS__); break;

template <int R, int TWO>
__device__ __forceinline__ void run_ops(float2 (&v)[1 << R], const DevOp* __restrict__ ops, int ob, int oe,
                                        const float2* __restrict__ coef, uint64_t gidx) {
  for (int o = ob; o < oe; ++o) {
    const DevOp op = ops[o];
    const bool gp = (gidx & op.gc) == op.gc;
    const unsigned rc = op.rc;
    const float2* c = coef + op.coef;
    switch (op.kind) {
      case DK_U1:
        switch (op.t0) { CASES_1(op_u1, v, c, rc, gp) }
        break;
      case DK_RY:
        switch (op.t0) { CASES_1(op_ry, v, c[0], rc, gp) }
        break;
      case DK_X:
        switch (op.t0) { CASES_1(op_x, v, rc, gp) }
        break;
      case DK_Y:
        switch (op.t0) { CASES_1(op_y, v, rc, gp) }
        break;
      case DK_DTAB:
        op_dtab<R>(v, op, c, gidx);
        break;
      case DK_KRY:
        op_kry<R>(v, c, op.t0);
        break;
      case DK_KU1:
        op_ku1<R>(v, c, op.t0);
        break;
      case DK_SCALE:
        op_scale<R>(v, c[0].x);
        break;
      case DK_U2:
        if constexpr (TWO) {
          switch (op.t0 * 8 + op.t1) { CASES_2(op_u2, v, c) }
        }
        break;
      case DK_CU2:
        if constexpr (TWO) {
          switch (op.t0 * 8 + op.t1) { CASES_2(op_cu2, v, c, rc, gp) }
        }
        break;
      case DK_SWAP:
        if constexpr (TWO) {
          switch (op.t0 * 8 + op.t1) { CASES_2(op_swap, v, rc, gp) }
        }
        break;
      case DK_XRY:
        if constexpr (TWO) {
          switch (op.t0 * 8 + op.t1) { CASES_2(op_xry, v, c) }
        }
        break;
      default:
        break;
    }
  }
}

// ------------------------------------------------------- noise blocks ------
// A noise block holds a run of consecutive stochastic channels (no gate in
// between) on at most 4 distinct qubits Q of a tile that is the whole state.
// Channel k's uniform is value k (= op.coef) of the item's seed stream.
// Every channel branch maps amplitudes as a'_i = c(bin(i)) * a_{i ^ m}, where
// bin(i) is the index's bits on Q and m flips bits of Q:
//   X: m = q, c = 1           Y: m = q, c = -i / +i (bit q clear / set)
//   Z: c = +1 / -1            no jump: c = r / sqrt(1-g) r, r = 1/sqrt(S0 + (1-g) S1)
//   damping jump: m = q, c = 1/sqrt(S1) / 0      dephasing jump: c = 0 / 1/sqrt(S1)
// (E1 of damping is [[0, sqrt g], [0, 0]], of dephasing [[0, 0], [0, sqrt l]],
// each renormalised exactly).  The form is closed under composition
// (C'(b) = c(b) C(b ^ m), M' = M ^ m), and so is the bin histogram of |a|^2
// (H'(b) = |c(b)|^2 H(b ^ m)).  So the block takes one histogram sweep (FP32
// squares summed in FP64; only when a damping or dephasing channel needs
// P(q=1)), decides every branch in order from the running histogram in FP64
// (damping / dephasing: jump when u < p1 = g S1 / (S0 + S1); depolarizing:
// the reference's ranges), and applies the composed map in one sweep
// (factors rounded to FP32 once).  Q is ascending (bin bit j = qubit Q[j]).
struct NoiseSmem {
  double red[16 * 16];  // per-warp bin sums (at most 16 warps per CTA)
  float2 C[16];        // composed factor per bin
  uint32_t M;          // composed flip mask over the bins (bit j = qubit Q[j])
  uint32_t identity;   // 1: the composed map is the identity
};

// Swizzled offsets of the 2^NQ bins: a tile index is base | off(b), with the
// Q bits of base clear, and phys is linear over GF(2), so
// phys(base | off(b)) = phys(base) ^ phys(off(b)).
template <int NQ>
__device__ __forceinline__ void bin_offsets(const int (&Q)[4], uint32_t (&poff)[1 << NQ]) {
#pragma unroll
  for (int b = 0; b < (1 << NQ); ++b) {
    uint32_t off = 0;
#pragma unroll
    for (int j = 0; j < NQ; ++j)
      if ((b >> j) & 1) off |= 1u << Q[j];
    poff[b] = phys(off);
  }
}

// Bin sums of |a|^2 (squares in FP32, sums in FP64; fixed order: per thread,
// then a warp butterfly) into red[warp * 16 + bin].  Q ascending.
template <int NQ>
__device__ __forceinline__ void noise_hist(const float2* tile, uint32_t N, const int (&Q)[4], double* red) {
  constexpr int NB = 1 << NQ;
  uint32_t poff[NB];
  bin_offsets<NQ>(Q, poff);
  double acc[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) acc[b] = 0.0;
  for (uint32_t r = threadIdx.x; r < (N >> NQ); r += blockDim.x) {
    uint32_t base = r;
#pragma unroll
    for (int j = 0; j < NQ; ++j) base = (uint32_t)insert_zero(base, Q[j]);
    const uint32_t pb = phys(base);
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const float2 a = tile[pb ^ poff[b]];
      acc[b] += (double)fmaf(a.x, a.x, __fmul_rn(a.y, a.y));
    }
  }
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    double v = acc[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[(threadIdx.x >> 5) * 16 + b] = v;
  }
}

// a'(base | off(b)) = C[b] * a(base | off(b ^ M)) over every base.
template <int NQ>
__device__ __forceinline__ void noise_apply(float2* tile, uint32_t N, const int (&Q)[4], const NoiseSmem* sm) {
  constexpr int NB = 1 << NQ;
  uint32_t poff[NB];
  bin_offsets<NQ>(Q, poff);
  const uint32_t M = sm->M;
  float2 Cv[NB], Cm[NB];  // C[b] and C[b ^ M]
#pragma unroll
  for (int b = 0; b < NB; ++b) { Cv[b] = sm->C[b]; Cm[b] = sm->C[b ^ M]; }
  for (uint32_t r = threadIdx.x; r < (N >> NQ); r += blockDim.x) {
    uint32_t base = r;
#pragma unroll
    for (int j = 0; j < NQ; ++j) base = (uint32_t)insert_zero(base, Q[j]);
    const uint32_t pb = phys(base);
    if (M == 0) {
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        float2& a = tile[pb ^ poff[b]];
        a = cmul(a, Cv[b]);
      }
    } else {
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int b2 = b ^ (int)M;
        if (b2 < b) continue;
        float2& ai = tile[pb ^ poff[b]];
        float2& aj = tile[pb ^ poff[b2]];
        const float2 vi = ai, vj = aj;
        ai = cmul(vj, Cv[b]);
        aj = cmul(vi, Cm[b]);
      }
    }
  }
}

// Warp 0: the branch of every channel of the block, in order, and the
// composed map.  Lane b < 2^nq holds bin b (its histogram entry and factor);
// sums over bins are xor butterflies, so every lane gets the same bits.  A
// branch's factor c(b) takes one of two values by bit q of the bin (lo for
// bit clear, hi for bit set).
__device__ __noinline__ void noise_decide(const DevOp* __restrict__ ops, int ob, int oe, const int (&Q)[4], int nq,
                                         bool have_h, int nw, uint64_t seed, uint8_t* nb, NoiseSmem* sm) {
  const int lane = threadIdx.x & 31;
  const int NB = 1 << nq;
  const bool mine = lane < NB;
  double H = 0.0, Cr = 1.0, Ci = 0.0;
  if (have_h && mine)
    for (int w = 0; w < nw; ++w) H += sm->red[w * 16 + lane];
  uint32_t mb = 0;
  bool ident = true;
  for (int o = ob; o < oe; ++o) {
    const DevOp op = ops[o];
    int j = 0;
    while (j < nq - 1 && Q[j] != op.t0) ++j;
    const int bit = 1 << j;
    const bool set = (lane & bit) != 0;
    const double g = __longlong_as_double((long long)op.gc);
    const double u = qs_seed_uniform_at(seed, op.coef);
    int m = 0;
    double cr = 1.0, ci = 0.0;
    if (op.d0 == QS_OP_DEPOLARIZE) {
      const int br = qs_depol_branch(g, u);
      if (lane == 0 && nb) nb[op.coef] = (uint8_t)br;
      if (br == 0) continue;
      if (br == 1) m = bit;
      else if (br == 2) { m = bit; cr = 0.0; ci = set ? 1.0 : -1.0; }
      else cr = set ? -1.0 : 1.0;
    } else {
      double s1 = set ? H : 0.0, s0 = set ? 0.0 : H;
#pragma unroll
      for (int x = 1; x < 16; x <<= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, x);
        s1 += __shfl_xor_sync(0xffffffffu, s1, x);
      }
      const double S0 = s0, S1 = s1;
      const double p1 = g * S1 / (S0 + S1);
      // the kept branch has norm^2 keep; a branch of zero weight is never taken
      const double keep = S0 + (1.0 - g) * S1;
      const bool jump = S1 > 0.0 && (u < p1 || !(keep > 0.0));
      if (lane == 0 && nb) nb[op.coef] = jump ? 1 : 0;
      if (!jump) {
        const double r = 1.0 / sqrt(keep);
        cr = set ? sqrt(1.0 - g) * r : r;
      } else if (op.d0 == QS_OP_AMP_DAMP) {
        m = bit;
        cr = set ? 0.0 : 1.0 / sqrt(S1);
      } else {
        cr = set ? 1.0 / sqrt(S1) : 0.0;
      }
    }
    ident = false;
    // C'(b) = c(b) C(b ^ m), H'(b) = |c(b)|^2 H(b ^ m)
    const double xr = __shfl_xor_sync(0xffffffffu, Cr, m), xi = __shfl_xor_sync(0xffffffffu, Ci, m);
    const double xh = __shfl_xor_sync(0xffffffffu, H, m);
    Cr = cr * xr - ci * xi;
    Ci = cr * xi + ci * xr;
    H = (cr * cr + ci * ci) * xh;
    mb ^= (uint32_t)m;
  }
  if (mine) sm->C[lane] = make_float2((float)Cr, (float)Ci);
  if (lane == 0) {
    sm->M = mb;
    sm->identity = ident ? 1u : 0u;
  }
}

__device__ __noinline__ void noise_block(float2* tile, int T, const DevBlock blk, const DevOp* __restrict__ ops,
                                        uint64_t seed, uint8_t* nb, NoiseSmem* sm) {
  const uint32_t N = 1u << T;
  const int nq = blk.pos[5];
  int Q[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) Q[j] = blk.pos[j];
  bool have_h = false;
  for (int o = blk.op_begin; o < blk.op_end; ++o) have_h |= ops[o].d0 != QS_OP_DEPOLARIZE;
  if (have_h) {
    switch (nq) {
      case 1: noise_hist<1>(tile, N, Q, sm->red); break;
      case 2: noise_hist<2>(tile, N, Q, sm->red); break;
      case 3: noise_hist<3>(tile, N, Q, sm->red); break;
      default: noise_hist<4>(tile, N, Q, sm->red); break;
    }
    __syncthreads();
  }
  if (threadIdx.x < 32)
    noise_decide(ops, blk.op_begin, blk.op_end, Q, nq, have_h, (int)(blockDim.x >> 5), seed, nb, sm);
  __syncthreads();
  if (sm->identity) return;
  switch (nq) {
    case 1: noise_apply<1>(tile, N, Q, sm); break;
    case 2: noise_apply<2>(tile, N, Q, sm); break;
    case 3: noise_apply<3>(tile, N, Q, sm); break;
    default: noise_apply<4>(tile, N, Q, sm); break;
  }
}

// Dense-4x4-only programs (TWO == 2: every op of every pass in the launch
// is an uncontrolled DK_U2, as in Quantum-Volume circuits): the op loop has
// no kind dispatch, no control predicates and none of the other ops' code,
// which keeps the register array's allocation across the pair switch
// simple.  Same arithmetic as run_ops, so the same bits.
template <int R>
__device__ __forceinline__ void run_ops_u2(float2 (&v)[1 << R], const DevOp* __restrict__ ops, int ob, int oe,
                                           const float2* __restrict__ coef) {
  for (int o = ob; o < oe; ++o) {
    const uchar4 k = *reinterpret_cast<const uchar4*>(ops + o);  // kind, t0, t1, rc
    const float2* c = coef + ops[o].coef;
    switch (k.y * 8 + k.z) { CASES_2(op_u2, v, c) }
  }
}

// One register block over the tile: every thread gathers the 2^R amplitudes
// of each of its groups (Gray-code walk over the swizzled addresses), runs
// the block's ops in registers and scatters them back.
template <int R, int TWO>
__device__ __forceinline__ void register_block(float2* tile, const DevBlock& blk, const DevOp* __restrict__ ops,
                                               const float2* __restrict__ s_coef, uint32_t ngroups, uint64_t gbase,
                                               const uint64_t* dep_lo, const uint64_t* dep_hi) {
  int pos[R];
  uint32_t pp[R];
#pragma unroll
  for (int k = 0; k < R; ++k) { pos[k] = blk.pos[k]; pp[k] = phys(1u << pos[k]); }
  const bool need_g = blk.pos[7] != 0;
  for (uint32_t g = threadIdx.x; g < ngroups; g += blockDim.x) {
    uint32_t base = g;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const uint32_t lo = base & ((1u << pos[k]) - 1u);
      base = ((base ^ lo) << 1) | lo;
    }
    const uint32_t pb = phys(base);
    const uint64_t gidx = need_g ? (gbase | dep_lo[base & 127] | dep_hi[base >> 7]) : 0ull;
    float2 v[1 << R];
    // Gray-code walk: consecutive indices differ in one register bit
    {
      uint32_t a = pb;
#pragma unroll
      for (int q = 0; q < (1 << R); ++q) {
        const int j = q ^ (q >> 1);
        if (q) a ^= pp[__ffs(q) - 1];
        v[j] = tile[a];
      }
    }
    if constexpr (TWO == 2) run_ops_u2<R>(v, ops, blk.op_begin, blk.op_end, s_coef);
    else run_ops<R, TWO>(v, ops, blk.op_begin, blk.op_end, s_coef, gidx);
    {
      uint32_t a = pb;
#pragma unroll
      for (int q = 0; q < (1 << R); ++q) {
        const int j = q ^ (q >> 1);
        if (q) a ^= pp[__ffs(q) - 1];
        tile[a] = v[j];
      }
    }
  }
}

// ---------------------------------------------------------- the kernel ----
// R = 5 keeps 32 amplitudes (64 registers) per thread: 128-thread CTAs, 3 per
// SM.  Narrower blocks use 256 threads.
constexpr int kMaxThreads(int R) { return R == 5 ? 128 : 256; }
constexpr int kMinBlocks(int R) { return R == 5 ? 2 : 2; }
// A 2^14-amplitude tile (128 KiB) leaves room for one CTA per SM; those
// launches use a variant with twice the threads (same register cap per
// thread) so that the SM still has 8-16 warps to switch between.
constexpr int kBigThreads(int R) { return 2 * kMaxThreads(R); }

// Dynamic shared memory: [tile 2^maxT float2][coefficient pool][dep tables].
template <int R, int TWO, bool BIG>
__global__ void __launch_bounds__(BIG ? kBigThreads(R) : kMaxThreads(R), BIG ? 1 : kMinBlocks(R))
k_pass(float2* __restrict__ base_state, PassItem single, const PassItem* __restrict__ items, int nitems,
       uint64_t total_tiles, uint32_t coef_off_bytes, uint32_t dep_off_bytes) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tile = reinterpret_cast<float2*>(smem_raw);
  float2* s_coef = reinterpret_cast<float2*>(smem_raw + coef_off_bytes);
  uint64_t* dep_lo = reinterpret_cast<uint64_t*>(smem_raw + dep_off_bytes);
  uint64_t* dep_hi = dep_lo + 128;
  int* s_S = reinterpret_cast<int*>(dep_hi + 128);
  __shared__ NoiseSmem s_noise;  // noise blocks

  int cur = -1;
  const DevPass* P = nullptr;
  float2* state = nullptr;
  int T = 0;

  for (uint64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    // Which item owns tile t (items sorted by tile_begin).
    int it = 0;
    if (nitems > 1) {
      int lo = 0, hi = nitems - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (items[mid].tile_begin <= t) lo = mid; else hi = mid - 1;
      }
      it = lo;
    }
    // A device table (even of one item) takes precedence over `single`.
    const PassItem I = items ? items[it] : single;
    if (it != cur) {
      __syncthreads();  // previous tables no longer in use
      cur = it;
      P = I.pass;
      state = base_state + I.state_off;
      T = P->T;
      if (threadIdx.x < 16) s_S[threadIdx.x] = P->S[threadIdx.x];
      const float2* gcoef = reinterpret_cast<const float2*>(reinterpret_cast<const char*>(P) + P->coef_off);
      for (uint32_t k = threadIdx.x; k < P->ncoef; k += blockDim.x) s_coef[k] = gcoef[k];
      __syncthreads();
      // dep(i) = sum_k bit_k(i) << S[k], split in two 7-bit tables.
      for (int e = threadIdx.x; e < 256; e += blockDim.x) {
        const int part = e >> 7, x = e & 127;
        uint64_t d = 0;
        for (int k = 0; k < 7; ++k) {
          const int kk = part * 7 + k;
          if (kk < T && ((x >> k) & 1)) d |= 1ull << s_S[kk];
        }
        if (part == 0) dep_lo[x] = d; else dep_hi[x] = d;
      }
      __syncthreads();
    }
    const uint64_t local = t - I.tile_begin;
    uint64_t gbase = local;
    for (int k = 0; k < T; ++k) gbase = insert_zero(gbase, s_S[k]);

    // 1. load the tile (pairs (2c, 2c+1) are adjacent in HBM: S[0] == 0)
    const uint32_t npairs = 1u << (T - 1);
    // |0..0>: only the tile holding index 0 of its state has a non-zero
    // entry (the bits above n_qubits select the state in a batch); every
    // other tile of a from-|0> pass stays +0 and skips the register blocks
    const bool zero_tile = (I.flags & PI_FROM_ZERO) && (gbase & ((1ull << P->n_qubits) - 1ull)) != 0ull;
    if (I.flags & PI_FROM_ZERO) {
      const bool first = !zero_tile;
      for (uint32_t c = threadIdx.x; c < npairs; c += blockDim.x) {
        const uint32_t i = c << 1;
        const float x = (first && i == 0) ? 1.f : 0.f;
        *reinterpret_cast<float4*>(tile + phys(i)) = make_float4(x, 0.f, 0.f, 0.f);
      }
    } else {
      for (uint32_t c = threadIdx.x; c < npairs; c += blockDim.x) {
        const uint32_t i = c << 1;
        const uint64_t g = gbase | dep_lo[i & 127] | dep_hi[i >> 7];
        cp_async16(tile + phys(i), state + g);
      }
      cp_async_wait_all();
    }
    __syncthreads();

    // 2. register blocks
    const DevBlock* blocks = reinterpret_cast<const DevBlock*>(reinterpret_cast<const char*>(P) + P->block_off);
    const DevOp* ops = reinterpret_cast<const DevOp*>(reinterpret_cast<const char*>(P) + P->op_off);
    const int nblocks = zero_tile ? 0 : P->nblocks;
    const uint32_t ngroups = 1u << (T - R);
    for (int b = 0; b < nblocks; ++b) {
      const DevBlock blk = blocks[b];
      if (blk.pos[6]) {  // noise block (only in programs whose tile is the whole state)
        noise_block(tile, T, blk, ops, I.noise_seed, I.noise_branch, &s_noise);
        __syncthreads();
        continue;
      }
      register_block<R, TWO>(tile, blk, ops, s_coef, ngroups, gbase, dep_lo, dep_hi);
      __syncthreads();
    }

    // 3. store the tile back in place
    for (uint32_t c = threadIdx.x; c < npairs; c += blockDim.x) {
      const uint32_t i = c << 1;
      const uint64_t g = gbase | dep_lo[i & 127] | dep_hi[i >> 7];
      *reinterpret_cast<float4*>(state + g) = *reinterpret_cast<const float4*>(tile + phys(i));
    }
    __syncthreads();
  }
}

// ------------------------------------------------- persistent batch kernel -
// Every (state, pass) item of a batch in one launch.  Items are numbered
// level by level (every state's first pass, then every second pass, ...) and
// their tiles consecutively; CTAs take tiles one at a time from a device
// counter in that order.  Before a tile of item i, the CTA waits until item
// pred(i) (PassItem.pred: the same state's previous pass) has stored all its
// tiles, counted per item.  Tiles are handed out in order and every CTA that
// holds one is running, so a wait only depends on tiles already taken by
// running CTAs.  Each wait is bounded (`limit` ns of %globaltimer): when it
// runs out the CTA ORs 4 into the status word and takes no further tile.
// `withhold` names an item whose tiles are not counted (a test hook; ~0u
// otherwise), so that the waits of its dependents run out.
constexpr uint32_t kNoPred = 0xffffffffu;

__device__ __forceinline__ uint64_t q_gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t q_ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <int R, int TWO>
__device__ __forceinline__ void queue_blocks(float2* tile, const DevPass* P, const float2* s_coef, uint64_t gbase,
                                             const uint64_t* dep_lo, const uint64_t* dep_hi) {
  const DevBlock* blocks = reinterpret_cast<const DevBlock*>(reinterpret_cast<const char*>(P) + P->block_off);
  const DevOp* ops = reinterpret_cast<const DevOp*>(reinterpret_cast<const char*>(P) + P->op_off);
  const uint32_t ngroups = 1u << (P->T - R);
  for (int b = 0; b < P->nblocks; ++b) {
    register_block<R, TWO>(tile, blocks[b], ops, s_coef, ngroups, gbase, dep_lo, dep_hi);
    __syncthreads();
  }
}

template <int TWO, bool BIG>
__global__ void __launch_bounds__(BIG ? 256 : 128, BIG ? 1 : 2)
k_pass_queue(float2* __restrict__ base_state, const PassItem* __restrict__ items, int nitems, uint64_t total_tiles,
             uint32_t coef_off_bytes, uint32_t dep_off_bytes, uint32_t* __restrict__ counters,
             uint32_t* __restrict__ status, uint64_t limit, uint32_t withhold) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tile = reinterpret_cast<float2*>(smem_raw);
  float2* s_coef = reinterpret_cast<float2*>(smem_raw + coef_off_bytes);
  uint64_t* dep_lo = reinterpret_cast<uint64_t*>(smem_raw + dep_off_bytes);
  uint64_t* dep_hi = dep_lo + 128;
  int* s_S = reinterpret_cast<int*>(dep_hi + 128);
  __shared__ unsigned long long s_task;
  __shared__ int s_fail;
  unsigned long long* next = reinterpret_cast<unsigned long long*>(counters);  // counters[0..1]
  uint32_t* done = counters + 2;
  int cur = -1;
  const DevPass* P = nullptr;
  for (;;) {
    if (threadIdx.x == 0) s_task = atomicAdd(next, 1ull);
    __syncthreads();
    const uint64_t t = s_task;
    if (t >= total_tiles) break;
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (items[mid].tile_begin <= t) lo = mid; else hi = mid - 1;
    }
    const int it = lo;
    const PassItem I = items[it];
    if (threadIdx.x == 0) {
      s_fail = 0;
      if (I.pred != kNoPred) {
        const uint32_t need = (uint32_t)items[I.pred].ntiles;
        if (q_ld_acquire(done + I.pred) < need) {
          const uint64_t t0 = q_gtimer();
          while (q_ld_acquire(done + I.pred) < need) {
            if (q_gtimer() - t0 > limit) {
              s_fail = 1;
              break;
            }
            __nanosleep(256);
          }
        }
      }
    }
    __syncthreads();
    if (s_fail) {
      if (threadIdx.x == 0) atomicOr(status, 4u);
      break;
    }
    if (it != cur) {
      cur = it;
      P = I.pass;
      if (threadIdx.x < 16) s_S[threadIdx.x] = P->S[threadIdx.x];
      const float2* gcoef = reinterpret_cast<const float2*>(reinterpret_cast<const char*>(P) + P->coef_off);
      for (uint32_t k = threadIdx.x; k < P->ncoef; k += blockDim.x) s_coef[k] = gcoef[k];
      __syncthreads();
      for (int e = threadIdx.x; e < 256; e += blockDim.x) {
        const int part = e >> 7, x = e & 127;
        uint64_t d = 0;
        for (int k = 0; k < 7; ++k) {
          const int kk = part * 7 + k;
          if (kk < P->T && ((x >> k) & 1)) d |= 1ull << s_S[kk];
        }
        if (part == 0) dep_lo[x] = d; else dep_hi[x] = d;
      }
      __syncthreads();
    }
    const int T = P->T;
    float2* state = base_state + I.state_off;
    uint64_t gbase = t - I.tile_begin;
    for (int k = 0; k < T; ++k) gbase = insert_zero(gbase, s_S[k]);
    const uint32_t npairs = 1u << (T - 1);
    const bool zero_tile = (I.flags & PI_FROM_ZERO) && (gbase & ((1ull << P->n_qubits) - 1ull)) != 0ull;
    if (I.flags & PI_FROM_ZERO) {
      for (uint32_t c = threadIdx.x; c < npairs; c += blockDim.x) {
        const uint32_t i = c << 1;
        const float x = (!zero_tile && i == 0) ? 1.f : 0.f;
        *reinterpret_cast<float4*>(tile + phys(i)) = make_float4(x, 0.f, 0.f, 0.f);
      }
    } else {
      for (uint32_t c = threadIdx.x; c < npairs; c += blockDim.x) {
        const uint32_t i = c << 1;
        const uint64_t g = gbase | dep_lo[i & 127] | dep_hi[i >> 7];
        cp_async16(tile + phys(i), state + g);
      }
      cp_async_wait_all();
    }
    __syncthreads();
    if (!zero_tile) {
      switch (P->R) {
        case 1: queue_blocks<1, TWO>(tile, P, s_coef, gbase, dep_lo, dep_hi); break;
        case 2: queue_blocks<2, TWO>(tile, P, s_coef, gbase, dep_lo, dep_hi); break;
        case 3: queue_blocks<3, TWO>(tile, P, s_coef, gbase, dep_lo, dep_hi); break;
        case 4: queue_blocks<4, TWO>(tile, P, s_coef, gbase, dep_lo, dep_hi); break;
        default: queue_blocks<5, TWO>(tile, P, s_coef, gbase, dep_lo, dep_hi); break;
      }
    }
    for (uint32_t c = threadIdx.x; c < npairs; c += blockDim.x) {
      const uint32_t i = c << 1;
      const uint64_t g = gbase | dep_lo[i & 127] | dep_hi[i >> 7];
      *reinterpret_cast<float4*>(state + g) = *reinterpret_cast<const float4*>(tile + phys(i));
    }
    __threadfence();   // this thread's stores, before the tile is counted
    __syncthreads();
    if (threadIdx.x == 0 && (uint32_t)it != withhold) atomicAdd(done + it, 1u);
  }
}

struct LaunchCfg { int per_sm; };

size_t coef_bytes_for(int ncoef) { return (((size_t)ncoef * sizeof(float2)) + 15) & ~size_t(15); }

// Launch shapes per (device, dynamic shared memory, threads).  Handles on
// several host threads launch concurrently, so the table is locked.
template <int R, int TWO, bool BIG>
LaunchCfg configure(int device, int smem, int threads) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, LaunchCfg> cache;
  static std::set<int> attr_set;
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_tuple(device, smem, threads);
  auto f = cache.find(key);
  if (f != cache.end()) return f->second;
  // The attribute is a per-function maximum on each device: set it once to
  // the largest tile (2^14 amplitudes) plus the largest coefficient pool, so
  // that launches of any size stay valid.
  if (!attr_set.count(device)) {
    QS_CUDA(cudaFuncSetAttribute(k_pass<R, TWO, BIG>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxPassSmem));
    attr_set.insert(device);
  }
  int per_sm = 0;
  QS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pass<R, TWO, BIG>, threads, smem));
  if (per_sm < 1) throw qs_error(QS_ERR_CUDA, "tile-pass kernel does not fit on an SM");
  LaunchCfg c{per_sm};
  cache[key] = c;
  return c;
}

template <int R, int TWO, bool BIG>
void launch_R(qs_context* h, float2* base, const PassItem& single, const PassItem* d_items, int nitems,
              uint64_t total, int maxT, int threads, int ncoef) {
  const uint32_t tile_bytes = (uint32_t)(sizeof(float2) << maxT);
  const uint32_t coef_off = tile_bytes;
  const uint32_t dep_off = coef_off + (uint32_t)coef_bytes_for(ncoef);
  const int smem = (int)(dep_off + 2 * 128 * sizeof(uint64_t) + 16 * sizeof(int));
  QS_CHECK_ARG(smem <= kMaxPassSmem, "tile-pass program too large for shared memory (coefficient pool)");
  LaunchCfg c = configure<R, TWO, BIG>(h->device, smem, threads);
  uint64_t grid = std::min<uint64_t>(total, (uint64_t)h->sm_count * c.per_sm);
  if (grid == 0) return;
  k_pass<R, TWO, BIG><<<(unsigned)grid, threads, smem, h->stream>>>(base, single, d_items, nitems, total,
                                                                    coef_off, dep_off);
  qs_after_launch(h, "k_pass");
}

// QSIM_BIG_TILES=0 keeps 14-qubit tiles on the default CTA size.
bool big_tiles_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("QSIM_BIG_TILES");
    return !(e && e[0] == '0');
  }();
  return on;
}

int threads_for(int maxT, int R) {
  const int cap = R == 5 ? 128 : 256;
  int groups = 1 << (maxT - R);
  int t = groups < cap ? groups : cap;
  if (t < 32) t = 32;
  return t;
}

template <int TWO>
void dispatch_two(qs_context* h, float2* base, const PassItem& single, const PassItem* d_items, int nitems,
                  uint64_t total, int maxT, int R, int ncoef, int threads_req) {
  int threads = threads_for(maxT, R);
  bool big = false;
  if (threads_req > 0) {
    threads = std::max(32, std::min(threads, threads_req));
  } else if (maxT >= 14 && R >= 2 && (1 << (maxT - R)) >= 2 * threads && big_tiles_enabled()) {
    threads *= 2;
    big = true;
  }
#define QS_LAUNCH_R(RR)                                                                      \
  (big ? launch_R<RR, TWO, true>(h, base, single, d_items, nitems, total, maxT, threads, ncoef) \
       : launch_R<RR, TWO, false>(h, base, single, d_items, nitems, total, maxT, threads, ncoef))
  switch (R) {
    case 1: launch_R<1, TWO, false>(h, base, single, d_items, nitems, total, maxT, threads, ncoef); break;
    case 2: QS_LAUNCH_R(2); break;
    case 3: QS_LAUNCH_R(3); break;
    case 4: QS_LAUNCH_R(4); break;
    case 5: QS_LAUNCH_R(5); break;
    default: throw qs_error(QS_ERR_INVALID, "register block width must be 1..5");
  }
#undef QS_LAUNCH_R
}

void dispatch(qs_context* h, float2* base, const PassItem& single, const PassItem* d_items, int nitems,
              uint64_t total, int maxT, int R, int has2, int ncoef, int threads_req = 0) {
  QS_CHECK_ARG(maxT >= 1 && maxT <= 14, "tile bits out of range");
  QS_CHECK_ARG(threads_req == 0 || (threads_req % 32) == 0, "threads per CTA must be a multiple of 32");
  if (has2 == 2) dispatch_two<2>(h, base, single, d_items, nitems, total, maxT, R, ncoef, threads_req);
  else if (has2) dispatch_two<1>(h, base, single, d_items, nitems, total, maxT, R, ncoef, threads_req);
  else dispatch_two<0>(h, base, single, d_items, nitems, total, maxT, R, ncoef, threads_req);
}

template <int TWO, bool BIG>
void launch_queue(qs_context* h, float2* base, const PassItem* d_items, int nitems, uint64_t total, int maxT,
                  int ncoef, uint32_t* counters, uint32_t withhold, uint64_t limit) {
  const int threads = BIG ? 256 : 128;
  const uint32_t tile_bytes = (uint32_t)(sizeof(float2) << maxT);
  const uint32_t coef_off = tile_bytes;
  const uint32_t dep_off = coef_off + (uint32_t)coef_bytes_for(ncoef);
  const int smem = (int)(dep_off + 2 * 128 * sizeof(uint64_t) + 16 * sizeof(int));
  QS_CHECK_ARG(smem <= kMaxPassSmem, "tile-pass program too large for shared memory (coefficient pool)");
  int per_sm = 0;
  {
    static std::mutex mu;
    static std::map<std::tuple<int, int>, int> cache;
    static std::set<int> attr_set;
    std::lock_guard<std::mutex> lk(mu);
    if (!attr_set.count(h->device)) {
      QS_CUDA(cudaFuncSetAttribute(k_pass_queue<TWO, BIG>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxPassSmem));
      attr_set.insert(h->device);
    }
    auto key = std::make_tuple(h->device, smem);
    auto f = cache.find(key);
    if (f != cache.end()) {
      per_sm = f->second;
    } else {
      QS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pass_queue<TWO, BIG>, threads, smem));
      if (per_sm < 1) throw qs_error(QS_ERR_CUDA, "persistent batch kernel does not fit on an SM");
      cache[key] = per_sm;
    }
  }
  // every CTA is resident at once (grid <= CTAs per SM x SMs): a CTA waiting
  // on a dependency only waits on tiles that running CTAs hold
  const uint64_t grid = std::min<uint64_t>(total, (uint64_t)h->sm_count * per_sm);
  if (grid == 0) return;
  QS_CUDA(cudaMemsetAsync(counters, 0, sizeof(uint32_t) * (2 + (size_t)nitems), h->stream));
  k_pass_queue<TWO, BIG><<<(unsigned)grid, threads, smem, h->stream>>>(base, d_items, nitems, total, coef_off, dep_off,
                                                                      counters, h->dev_status, limit, withhold);
  qs_after_launch(h, "k_pass_queue");
}

// ------------------------------------------- dense block matrices (TC) ---
// The tensor-core pass (qs_pass_tc.cu) applies each register block of a
// dense-4x4-only pass as one 32x32 complex matrix.  Thread j of a job runs
// the block's ops on the basis vector e_j with the interpreter's own op loop,
// which yields column j of the block matrix U; the real form
//   Bt[2i][2j] = Re U_ij, Bt[2i][2j+1] = -Im U_ij, Bt[2i+1][2j] = Im U_ij,
//   Bt[2i+1][2j+1] = Re U_ij        (row n = output, column k = input)
// is written split into its nearest TF32 value and the FP32 remainder, each
// as a 64 x 64 K-major operand in the no-swizzle canonical layout of
// tcgen05.mma (8-row groups of 2048 bytes, 16-byte K chunks 128 bytes apart).
__device__ __forceinline__ uint32_t tc_kmajor(uint32_t r, uint32_t k) {
  return ((r >> 3) * 2048u + (k >> 2) * 128u + (r & 7u) * 16u + (k & 3u) * 4u) >> 2;
}
__device__ __forceinline__ void tc_put(float* hi, float* lo, uint32_t n, uint32_t k, float x) {
  const float h = __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);  // nearest TF32
  const uint32_t e = tc_kmajor(n, k);
  hi[e] = h;
  lo[e] = x - h;
}

__global__ void __launch_bounds__(32) k_block_mats(const TcMatJob* __restrict__ jobs) {
  const TcMatJob J = jobs[blockIdx.x];
  const DevPass* P = J.pass;
  const DevBlock blk = reinterpret_cast<const DevBlock*>(reinterpret_cast<const char*>(P) + P->block_off)[J.block];
  const DevOp* ops = reinterpret_cast<const DevOp*>(reinterpret_cast<const char*>(P) + P->op_off);
  const float2* coef = reinterpret_cast<const float2*>(reinterpret_cast<const char*>(P) + P->coef_off);
  const uint32_t j = threadIdx.x;
  float2 v[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = make_float2(k == (int)j ? 1.f : 0.f, 0.f);
  run_ops_u2<5>(v, ops, blk.op_begin, blk.op_end, coef);
  float* hi = J.out;
  float* lo = J.out + 4096;
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    tc_put(hi, lo, 2 * i, 2 * j, v[i].x);
    tc_put(hi, lo, 2 * i, 2 * j + 1, -v[i].y);
    tc_put(hi, lo, 2 * i + 1, 2 * j, v[i].y);
    tc_put(hi, lo, 2 * i + 1, 2 * j + 1, v[i].x);
  }
}

}  // namespace

// One state, one pass: the item is passed by value (no device table), so the
// launch can be captured in a CUDA graph.
void qs_launch_pass_single(qs_context* h, void* state, const DevPass* d_pass, int T, int R, uint64_t ntiles,
                           uint32_t flags, int has2, int ncoef) {
  PassItem it{};
  it.state_off = 0;
  it.pass = d_pass;
  it.ntiles = ntiles;
  it.tile_begin = 0;
  it.flags = flags;
  dispatch(h, (float2*)state, it, nullptr, 1, ntiles, T, R, has2, ncoef);
}

// Several (state, pass) items in one launch; d_items is a caller-owned device
// table whose tile_begin fields hold the prefix sums of ntiles.
void qs_launch_pass_items(qs_context* h, void* base, const PassItem* d_items, int n_items, uint64_t total_tiles,
                          int maxT, int R, int has2, int ncoef, int threads) {
  if (n_items <= 0 || total_tiles == 0) return;
  PassItem dummy{};
  dispatch(h, (float2*)base, dummy, d_items, n_items, total_tiles, maxT, R, has2, ncoef, threads);
}

// The whole batch in one persistent launch (k_pass_queue): d_items holds the
// items level by level with tile_begin prefix sums and pred links; counters
// is a device buffer of 2 + n_items words (zeroed here, stream-ordered).
void qs_launch_pass_queue(qs_context* h, void* base, const PassItem* d_items, int n_items, uint64_t total_tiles,
                          int maxT, int has2, int ncoef, uint32_t* counters, uint32_t withhold, uint64_t limit_ns) {
  if (n_items <= 0 || total_tiles == 0) return;
  QS_CHECK_ARG(maxT >= 1 && maxT <= 14, "tile bits out of range");
  const bool big = maxT >= 14;
  float2* b = static_cast<float2*>(base);
  if (has2 == 2) {
    if (big) launch_queue<2, true>(h, b, d_items, n_items, total_tiles, maxT, ncoef, counters, withhold, limit_ns);
    else launch_queue<2, false>(h, b, d_items, n_items, total_tiles, maxT, ncoef, counters, withhold, limit_ns);
  } else if (has2) {
    if (big) launch_queue<1, true>(h, b, d_items, n_items, total_tiles, maxT, ncoef, counters, withhold, limit_ns);
    else launch_queue<1, false>(h, b, d_items, n_items, total_tiles, maxT, ncoef, counters, withhold, limit_ns);
  } else {
    if (big) launch_queue<0, true>(h, b, d_items, n_items, total_tiles, maxT, ncoef, counters, withhold, limit_ns);
    else launch_queue<0, false>(h, b, d_items, n_items, total_tiles, maxT, ncoef, counters, withhold, limit_ns);
  }
}

// Block matrices of dense-4x4-only R = 5 passes for the tensor-core pass:
// one 32-thread CTA per job, each writing 32 KiB at job.out.
void qs_launch_block_mats(qs_context* h, cudaStream_t stream, const TcMatJob* d_jobs, int n_jobs) {
  if (n_jobs <= 0) return;
  for (int b = 0; b < n_jobs; b += 65535) {
    const int n = std::min(65535, n_jobs - b);
    k_block_mats<<<n, 32, 0, stream>>>(d_jobs + b);
    qs_after_launch(h, "k_block_mats");
  }
}
