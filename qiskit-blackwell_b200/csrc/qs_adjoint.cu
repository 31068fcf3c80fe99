// qs_adjoint.cu — adjoint-method gradient of E(theta) = <psi|H|psi>.
//
// Method (Jones & Gacon, "Efficient calculation of gradients in classical
// simulations of variational quantum algorithms", arXiv:2009.02823):
//   psi = U_L..U_1|0>,  lam = H psi,  E = Re<psi|lam>;
//   for l = L..1:  if U_l = exp(-i theta G/2):  dE/dtheta += Im<lam|G|psi>
//                  psi <- U_l^dag psi,  lam <- U_l^dag lam.
// (2 Re<lam| dU/dtheta |psi_{l-1}> = 2 Re(-i/2 <lam|G U psi_{l-1}>) = Im<lam|G|psi_l>.)
//
// The forward pass uses the batch planner (all parameter vectors in one set
// of tile-pass launches).  The reverse sweep is cut into tile passes too:
// consecutive (reversed) gates whose targets fit one tile of T qubits (the
// low qubits plus those the gates touch; controls may lie anywhere) run in one
// launch over all tiles of all parameter vectors.  A CTA stages the tile of
// both psi and lam in shared memory, applies every gate's U^dag there and, for
// each parameter gate, writes its FP64 partial of Im<lam|G|psi> (taken before
// the gate is undone); a final kernel sums the partials in a fixed order
// (deterministic).  So psi and lam cross HBM once per pass instead of once per
// gate.  QSIM_ADJ_PASSES=0 selects the older one-launch-per-gate sweep (kept
// for comparison; same arithmetic per gate, different summation order).
// There is no reference counterpart (ROADMAP.md:173-175 lists adjoint
// differentiation as future work).
#include "qs_api.h"
#include "qs_common.cuh"
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <set>

using namespace qs;

void* qs_upload_terms(qs_context* h, size_t offset, int n, const uint64_t* x, const uint64_t* z, const double* c,
                      int nterms);

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = 0.0;
  if (w == 0) { v = lane < nw ? ws[lane] : 0.0; v = warp_sum(v); }
  return v;
}

// Per-vector slicing along grid.x.
struct Slice { int nbx; uint64_t per; };
Slice slice(uint64_t items) {
  uint64_t nb = (items + 8191) / 8192;
  if (nb > 256) nb = 256;
  if (nb < 1) nb = 1;
  return Slice{(int)nb, (items + nb - 1) / nb};
}

struct Mat2 { float2 g[4]; };

// One 2x2 gate U^dag on both psi and lam of every vector b; if gkind != 0,
// partial[b][bx] = sum Im(<lam|G|psi>) over this block's pairs (before U^dag).
__global__ void k_adj_1q(float2* __restrict__ base, uint64_t vstride, uint64_t npairs, int t,
                         const Mat2* __restrict__ udag, int gkind, uint64_t per, double* __restrict__ partial) {
  const int b = blockIdx.y;
  float2* psi = base + (uint64_t)b * vstride;
  float2* lam = psi + (vstride / 3);
  const Mat2 U = udag[b];
  const uint64_t st = 1ull << t;
  const uint64_t p0 = (uint64_t)blockIdx.x * per, pe = min(p0 + per, npairs);
  double acc = 0.0;
  for (uint64_t p = p0 + threadIdx.x; p < pe; p += blockDim.x) {
    const uint64_t i0 = insert_zero(p, t), i1 = i0 | st;
    float2 a0 = psi[i0], a1 = psi[i1], l0 = lam[i0], l1 = lam[i1];
    if (gkind) {
      // (G psi) on the pair
      float2 g0, g1;
      if (gkind == 1) { g0 = a1; g1 = a0; }                                          // X
      else if (gkind == 2) { g0 = make_float2(a1.y, -a1.x); g1 = make_float2(-a0.y, a0.x); }  // Y
      else { g0 = a0; g1 = make_float2(-a1.x, -a1.y); }                             // Z
      // Im(conj(l) * g) = l.x*g.y - l.y*g.x
      acc += (double)l0.x * g0.y - (double)l0.y * g0.x + (double)l1.x * g1.y - (double)l1.y * g1.x;
    }
    psi[i0] = cfma2(U.g[0], a0, U.g[1], a1);
    psi[i1] = cfma2(U.g[2], a0, U.g[3], a1);
    lam[i0] = cfma2(U.g[0], l0, U.g[1], l1);
    lam[i1] = cfma2(U.g[2], l0, U.g[3], l1);
  }
  if (gkind) {
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[(uint64_t)b * gridDim.x + blockIdx.x] = acc;
  }
}

struct Mat4 { float2 g[16]; };
__global__ void k_adj_2q(float2* __restrict__ base, uint64_t vstride, uint64_t nquads, int q0, int q1, Mat4 U) {
  const int b = blockIdx.y;
  float2* psi = base + (uint64_t)b * vstride;
  float2* lam = psi + (vstride / 3);
  const int lo = min(q0, q1), hi = max(q0, q1);
  const uint64_t s0 = 1ull << q0, s1 = 1ull << q1;
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nquads; p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = insert_zero(insert_zero(p, lo), hi);
    float2* vs[2] = {psi, lam};
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      float2* s = vs[v];
      float2 a0 = s[i], a1 = s[i | s0], a2 = s[i | s1], a3 = s[i | s0 | s1];
      s[i] = cfma4(U.g + 0, a0, a1, a2, a3);
      s[i | s0] = cfma4(U.g + 4, a0, a1, a2, a3);
      s[i | s1] = cfma4(U.g + 8, a0, a1, a2, a3);
      s[i | s0 | s1] = cfma4(U.g + 12, a0, a1, a2, a3);
    }
  }
}

struct SortedQ { int pos[10]; int k; };
__global__ void k_adj_mcx(float2* __restrict__ base, uint64_t vstride, uint64_t items, SortedQ P, uint64_t cmask,
                          int t) {
  const int b = blockIdx.y;
  float2* psi = base + (uint64_t)b * vstride;
  float2* lam = psi + (vstride / 3);
  const uint64_t st = 1ull << t;
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < items; p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = insert_zeros(p, P.pos, P.k) | cmask;
    float2 a = psi[i0], c = psi[i0 | st];
    psi[i0] = c; psi[i0 | st] = a;
    a = lam[i0]; c = lam[i0 | st];
    lam[i0] = c; lam[i0 | st] = a;
  }
}

__global__ void k_adj_phase(float2* __restrict__ base, uint64_t vstride, uint64_t items, SortedQ P, uint64_t mask,
                            float2 ph, int neg) {
  const int b = blockIdx.y;
  float2* psi = base + (uint64_t)b * vstride;
  float2* lam = psi + (vstride / 3);
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < items; p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = insert_zeros(p, P.pos, P.k) | mask;
    float2 a = psi[i], l = lam[i];
    if (neg) { psi[i] = make_float2(-a.x, -a.y); lam[i] = make_float2(-l.x, -l.y); }
    else { psi[i] = cmul_comp(a, ph); lam[i] = cmul_comp(l, ph); }
  }
}

// E_b partials: Re<psi|lam>
__global__ void k_adj_dot(const float2* __restrict__ base, uint64_t vstride, uint64_t n, uint64_t per,
                          double* __restrict__ partial) {
  const int b = blockIdx.y;
  const float2* psi = base + (uint64_t)b * vstride;
  const float2* lam = psi + (vstride / 3);
  const uint64_t i0 = (uint64_t)blockIdx.x * per, e = min(i0 + per, n);
  double acc = 0.0;
  for (uint64_t i = i0 + threadIdx.x; i < e; i += blockDim.x) {
    const float2 a = psi[i], l = lam[i];
    acc += (double)a.x * l.x + (double)a.y * l.y;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[(uint64_t)b * gridDim.x + blockIdx.x] = acc;
}

// out[b*ostride + idx] (+)= sum_x partial[b][x], fixed order
__global__ void k_adj_final(const double* __restrict__ partial, int nbx, double* __restrict__ out, int ostride,
                            int idx, int add) {
  const int b = blockIdx.x;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nbx; i += blockDim.x) acc += partial[(uint64_t)b * nbx + i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) {
    double* o = out + (uint64_t)b * ostride + idx;
    *o = add ? (*o + acc) : acc;
  }
}

// k_pauli_apply equivalent per vector: lam = H psi (defined in qs_reduce.cu
// for a single state; re-stated here for the strided batch layout).
struct TermL { uint64_t x, z; double wr, wi; };
__global__ void k_adj_hpsi(float2* __restrict__ base, uint64_t vstride, uint64_t n, const TermL* __restrict__ terms,
                           int nterms) {
  extern __shared__ TermL st[];
  for (int k = threadIdx.x; k < nterms; k += blockDim.x) st[k] = terms[k];
  __syncthreads();
  const int b = blockIdx.y;
  const float2* psi = base + (uint64_t)b * vstride;
  float2* lam = base + (uint64_t)b * vstride + (vstride / 3);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nterms; ++k) {
      const TermL T = st[k];
      const uint64_t j = i ^ T.x;
      const float2 v = psi[j];
      const double sg = (__popcll(j & T.z) & 1) ? -1.0 : 1.0;
      re += sg * (T.wr * v.x - T.wi * v.y);
      im += sg * (T.wr * v.y + T.wi * v.x);
    }
    lam[i] = make_float2((float)re, (float)im);
  }
}

// ------------------------------------------------ reverse-sweep passes ----
enum AdjKind : int32_t { AG_1Q = 1, AG_MCX = 2, AG_PHASE = 3, AG_U2 = 4 };

struct AdjGate {
  int32_t kind;
  int32_t p0, p1;     // tile positions of the target(s); U2: p0 = matrix bit 0
  int32_t gkind;      // 1Q parameter gate generator: 1 X, 2 Y, 3 Z; 0 none
  int32_t slot;       // partial-sum slot of a parameter gate, else -1
  int32_t mat;        // 1Q: op index into the per-(op, vector) U^dag table; U2: Mat4 index
  int32_t neg;        // phase: negate instead of multiplying
  int32_t pad;
  uint64_t cmask;     // MCX controls / phase qubits, as a global index mask
  float2 ph;          // phase factor (already conjugated)
  float2 pad2;
};

struct PassArg {
  int32_t S[16];      // tile positions (global qubits), ascending
  int32_t T;
  int32_t gb, ge;     // gate range of the pass
  int32_t nslots;     // parameter-gate slots of the whole sweep
  int32_t from_zero;  // forward: the tile starts as |0..0> instead of being loaded
  int32_t pad[3];
};

__device__ __forceinline__ double block_sum_fixed(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
  __syncthreads();
  return t;  // valid on thread 0
}

__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// One pass: CTA (tile, vector b).  Reverse (FWD false): psi and lam tiles
// staged, every gate's U^dag applied to both, parameter-gate partials
// written.  Forward (FWD true): psi only, every gate's U applied (the
// conjugate transpose of the stored U^dag), from |0..0> when P.from_zero.
// Shared memory: psi tile, lam tile (reverse only; 2^T float2 each), then the
// 2 x 128 dep tables.
template <bool FWD>
__global__ void __launch_bounds__(kThreads) k_adj_pass(float2* __restrict__ base, uint64_t vstride, PassArg P,
                                                      const AdjGate* __restrict__ gates,
                                                      const Mat2* __restrict__ udag, int nb,
                                                      const Mat4* __restrict__ u2, double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char adj_smem[];
  const int T = P.T;
  const uint32_t NT = 1u << T;
  float2* sp = reinterpret_cast<float2*>(adj_smem);
  float2* sl = FWD ? sp : sp + NT;
  uint64_t* dep_lo = reinterpret_cast<uint64_t*>(sp + (FWD ? NT : 2 * NT));
  uint64_t* dep_hi = dep_lo + 128;
  __shared__ double red[kThreads / 32];
  const int b = blockIdx.y;
  const uint64_t tile = blockIdx.x, ntiles = gridDim.x;
  float2* psi = base + (uint64_t)b * vstride;
  float2* lam = psi + (vstride / 3);
  for (int e = threadIdx.x; e < 256; e += blockDim.x) {
    const int part = e >> 7, x = e & 127;
    uint64_t d = 0;
    for (int k = 0; k < 7; ++k) {
      const int kk = part * 7 + k;
      if (kk < T && ((x >> k) & 1)) d |= 1ull << P.S[kk];
    }
    if (part == 0) dep_lo[x] = d; else dep_hi[x] = d;
  }
  uint64_t gbase = tile;
  for (int k = 0; k < T; ++k) gbase = insert_zero(gbase, P.S[k]);
  __syncthreads();
  auto gidx = [&](uint32_t i) { return gbase | dep_lo[i & 127] | dep_hi[i >> 7]; };
  if (FWD && P.from_zero) {
    const bool first = gbase == 0;
    for (uint32_t i = threadIdx.x; i < NT; i += blockDim.x) sp[i] = make_float2(first && i == 0 ? 1.f : 0.f, 0.f);
  } else {
    for (uint32_t i = threadIdx.x; i < NT; i += blockDim.x) {
      const uint64_t g = gidx(i);
      sp[i] = psi[g];
      if (!FWD) sl[i] = lam[g];
    }
  }
  __syncthreads();
  for (int gi = P.gb; gi < P.ge; ++gi) {
    const AdjGate G = gates[gi];
    if (G.kind == AG_1Q) {
      Mat2 U = udag[(uint64_t)G.mat * nb + b];
      if (FWD) {
        const float2 u1 = U.g[1];
        U.g[0] = conjf2(U.g[0]);
        U.g[1] = conjf2(U.g[2]);
        U.g[2] = conjf2(u1);
        U.g[3] = conjf2(U.g[3]);
      }
      const int p = G.p0;
      double acc = 0.0;
      for (uint32_t c = threadIdx.x; c < (NT >> 1); c += blockDim.x) {
        const uint32_t i0 = (uint32_t)insert_zero(c, p), i1 = i0 | (1u << p);
        const float2 a0 = sp[i0], a1 = sp[i1];
        if (FWD) {
          sp[i0] = cfma2(U.g[0], a0, U.g[1], a1);
          sp[i1] = cfma2(U.g[2], a0, U.g[3], a1);
          continue;
        }
        const float2 l0 = sl[i0], l1 = sl[i1];
        if (G.gkind) {
          float2 g0, g1;
          if (G.gkind == 1) { g0 = a1; g1 = a0; }
          else if (G.gkind == 2) { g0 = make_float2(a1.y, -a1.x); g1 = make_float2(-a0.y, a0.x); }
          else { g0 = a0; g1 = make_float2(-a1.x, -a1.y); }
          acc += (double)l0.x * g0.y - (double)l0.y * g0.x + (double)l1.x * g1.y - (double)l1.y * g1.x;
        }
        sp[i0] = cfma2(U.g[0], a0, U.g[1], a1);
        sp[i1] = cfma2(U.g[2], a0, U.g[3], a1);
        sl[i0] = cfma2(U.g[0], l0, U.g[1], l1);
        sl[i1] = cfma2(U.g[2], l0, U.g[3], l1);
      }
      if (!FWD && G.slot >= 0) {
        const double t = block_sum_fixed(acc, red);
        if (threadIdx.x == 0) partial[((uint64_t)b * P.nslots + G.slot) * ntiles + tile] = t;
      }
    } else if (G.kind == AG_MCX) {
      const int p = G.p0;
      for (uint32_t c = threadIdx.x; c < (NT >> 1); c += blockDim.x) {
        const uint32_t i0 = (uint32_t)insert_zero(c, p), i1 = i0 | (1u << p);
        if ((gidx(i0) & G.cmask) != G.cmask) continue;
        const float2 a0 = sp[i0];
        sp[i0] = sp[i1];
        sp[i1] = a0;
        if (!FWD) {
          const float2 l0 = sl[i0];
          sl[i0] = sl[i1];
          sl[i1] = l0;
        }
      }
    } else if (G.kind == AG_PHASE) {
      const float2 ph = FWD ? conjf2(G.ph) : G.ph;
      for (uint32_t i = threadIdx.x; i < NT; i += blockDim.x) {
        if ((gidx(i) & G.cmask) != G.cmask) continue;
        const float2 a = sp[i];
        sp[i] = G.neg ? make_float2(-a.x, -a.y) : cmul_comp(a, ph);
        if (!FWD) {
          const float2 l = sl[i];
          sl[i] = G.neg ? make_float2(-l.x, -l.y) : cmul_comp(l, ph);
        }
      }
    } else {  // AG_U2
      Mat4 U = u2[G.mat];
      if (FWD) {
        const Mat4 D = U;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) U.g[4 * r + c] = conjf2(D.g[4 * c + r]);
      }
      const int lo = min(G.p0, G.p1), hi = max(G.p0, G.p1);
      const uint32_t s0 = 1u << G.p0, s1 = 1u << G.p1;
      for (uint32_t c = threadIdx.x; c < (NT >> 2); c += blockDim.x) {
        const uint32_t i = (uint32_t)insert_zero(insert_zero(c, lo), hi);
        float2* vs[2] = {sp, sl};
#pragma unroll
        for (int v = 0; v < (FWD ? 1 : 2); ++v) {
          float2* x = vs[v];
          const float2 a0 = x[i], a1 = x[i | s0], a2 = x[i | s1], a3 = x[i | s0 | s1];
          x[i] = cfma4(U.g + 0, a0, a1, a2, a3);
          x[i | s0] = cfma4(U.g + 4, a0, a1, a2, a3);
          x[i | s1] = cfma4(U.g + 8, a0, a1, a2, a3);
          x[i | s0 | s1] = cfma4(U.g + 12, a0, a1, a2, a3);
        }
      }
    }
    __syncthreads();
  }
  for (uint32_t i = threadIdx.x; i < NT; i += blockDim.x) {
    const uint64_t g = gidx(i);
    psi[g] = sp[i];
    if (!FWD) lam[g] = sl[i];
  }
}

// grads[b][param_of[s]] += sum over tiles of partial[b][s][tile], slots in
// order, tiles in order (deterministic).
__global__ void k_adj_slots(const double* __restrict__ partial, int nslots, uint64_t ntiles,
                            const int32_t* __restrict__ param_of, double* __restrict__ grads, int nparams) {
  __shared__ double red[kThreads / 32];
  const int b = blockIdx.x;
  for (int sidx = 0; sidx < nslots; ++sidx) {
    double acc = 0.0;
    const double* p = partial + ((uint64_t)b * nslots + sidx) * ntiles;
    for (uint64_t t = threadIdx.x; t < ntiles; t += blockDim.x) acc += p[t];
    const double t = block_sum_fixed(acc, red);
    if (threadIdx.x == 0) grads[(uint64_t)b * nparams + param_of[sidx]] += t;
  }
}

SortedQ sortedq(std::vector<int> q) {
  std::sort(q.begin(), q.end());
  SortedQ P;
  std::memset(&P, 0, sizeof(P));
  P.k = (int)q.size();
  for (int i = 0; i < P.k; ++i) P.pos[i] = q[i];
  return P;
}

using cd = std::complex<double>;

// 2x2 matrix of a rotation / U1 / DIAG1 op with parameter theta
void mat_1q(const qs_op& o, double theta, cd* m) {
  const double c = std::cos(theta / 2), s = std::sin(theta / 2);
  switch (o.kind) {
    case QS_OP_RX: m[0] = c; m[1] = cd(0, -s); m[2] = cd(0, -s); m[3] = c; break;
    case QS_OP_RY: m[0] = c; m[1] = -s; m[2] = s; m[3] = c; break;
    case QS_OP_RZ: m[0] = std::polar(1.0, -theta / 2); m[1] = 0; m[2] = 0; m[3] = std::polar(1.0, theta / 2); break;
    case QS_OP_U1: for (int i = 0; i < 4; ++i) m[i] = cd(o.m[2 * i], o.m[2 * i + 1]); break;
    case QS_OP_DIAG1: m[0] = cd(o.m[0], o.m[1]); m[1] = 0; m[2] = 0; m[3] = cd(o.m[2], o.m[3]); break;
    case QS_OP_Y: m[0] = 0; m[1] = cd(0, -1); m[2] = cd(0, 1); m[3] = 0; break;
    default: throw qs_error(QS_ERR_INVALID, "internal: not a 1Q op");
  }
}

// Reverse-sweep tile width: two staged vectors of 2^12 complex64 = 64 KiB.
constexpr int kAdjTileBits = 12;

bool adj_passes_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("QSIM_ADJ_PASSES");
    return !(e && e[0] == '0');
  }();
  return on;
}

bool is_1q_kind(int k) {
  return k == QS_OP_RX || k == QS_OP_RY || k == QS_OP_RZ || k == QS_OP_U1 || k == QS_OP_DIAG1 || k == QS_OP_Y;
}

}  // namespace

extern "C" int qs_adjoint_gradient(qs_handle_t h, int n, const qs_op* ops, int nops, int nparams,
                                   const double* params, int nb, const uint64_t* xm, const uint64_t* zm,
                                   const double* coefs, int nterms, void* work, double* energies, double* grads) {
  QS_REQUIRE_HANDLE(h);
  qs_batch_plan_t fwd = nullptr;
  void* dbuf = nullptr;
  void* pbuf = nullptr;
  QS_API_BEGIN
  qs_check_state(work, n);
  QS_CHECK_ARG(nb >= 1 && nb <= 65535, "n_batch must be in [1, 65535]");
  QS_CHECK_ARG(nparams >= 0 && (nparams == 0 || params), "bad params");
  QS_CHECK_ARG(nops >= 1 && ops, "need at least one op");
  QS_CHECK_ARG(nterms >= 1 && nterms <= 1024, "n_terms must be in [1, 1024]");
  QS_CHECK_ARG(energies && grads, "null output pointers");
  const uint64_t N = 1ull << n;
  const uint64_t vstride = 3 * N;
  for (int i = 0; i < nops; ++i)
    if (ops[i].param >= nparams) throw qs_error(QS_ERR_INVALID, "op param index out of range");

  for (int i = 0; i < nops; ++i) {
    const qs_op& o = ops[i];
    if (o.param >= 0 && is_1q_kind(o.kind))
      QS_CHECK_ARG(o.kind == QS_OP_RX || o.kind == QS_OP_RY || o.kind == QS_OP_RZ,
                   "only RX/RY/RZ ops may carry a parameter");
    QS_CHECK_ARG(is_1q_kind(o.kind) || o.kind == QS_OP_MCX || o.kind == QS_OP_MCPHASE || o.kind == QS_OP_U2,
                 "op kind not supported by the adjoint sweep");
  }
  // The pass sweeps keep one FP64 partial per (vector, parameter gate, tile);
  // past 1 GiB of partials the per-gate sweep (partials per block) is used.
  size_t n_param_gates = 0;
  for (int i = 0; i < nops; ++i) n_param_gates += (ops[i].param >= 0 && is_1q_kind(ops[i].kind)) ? 1 : 0;
  const int T = std::min(n, kAdjTileBits);
  const uint64_t ntiles = 1ull << (n - T);
  const bool use_passes = adj_passes_enabled() &&
      (double)nb * (double)std::max<size_t>(n_param_gates, 1) * (double)ntiles * sizeof(double) <=
          (double)(1ull << 30);

  // device buffer: grads [nb][nparams] | energies [nb] | partial [nb][256] | U^dag tables
  const size_t ng = (size_t)nb * std::max(nparams, 1);
  const Slice sl = slice(N / 2);
  const Slice sd = slice(N);
  const int nbx = std::max(sl.nbx, sd.nbx);
  size_t bytes = sizeof(double) * (ng + nb + (size_t)nb * nbx) + sizeof(Mat2) * (size_t)nb * nops + 64;
  QS_CUDA(cudaMallocAsync(&dbuf, bytes, h->stream));
  double* d_grads = (double*)dbuf;
  double* d_energy = d_grads + ng;
  double* d_part = d_energy + nb;
  Mat2* d_udag = (Mat2*)(((uintptr_t)(d_part + (size_t)nb * nbx) + 15) & ~uintptr_t(15));
  QS_CUDA(cudaMemsetAsync(d_grads, 0, sizeof(double) * ng, h->stream));

  // per-(op, b) U^dag for the 1Q ops
  std::vector<Mat2> udag((size_t)nb * nops);
  for (int i = 0; i < nops; ++i) {
    if (!is_1q_kind(ops[i].kind)) continue;
    for (int b = 0; b < nb; ++b) {
      const double th = ops[i].param >= 0 ? params[(size_t)b * nparams + ops[i].param] : ops[i].m[0];
      cd m[4];
      mat_1q(ops[i], th, m);
      Mat2& U = udag[(size_t)i * nb + b];
      // conjugate transpose
      U.g[0] = make_float2((float)m[0].real(), (float)-m[0].imag());
      U.g[1] = make_float2((float)m[2].real(), (float)-m[2].imag());
      U.g[2] = make_float2((float)m[1].real(), (float)-m[1].imag());
      U.g[3] = make_float2((float)m[3].real(), (float)-m[3].imag());
    }
  }
  QS_CUDA(cudaMemcpyAsync(d_udag, udag.data(), sizeof(Mat2) * udag.size(), cudaMemcpyHostToDevice, h->stream));

  // ---- tile passes (forward order and reverse order)
  std::vector<AdjGate> gates;
  std::vector<PassArg> fpasses, rpasses;
  std::vector<int32_t> param_of;
  std::vector<Mat4> u2s;
  AdjGate* d_gates = nullptr;
  Mat4* d_u2 = nullptr;
  int32_t* d_param_of = nullptr;
  double* d_parts = nullptr;
  size_t pass_smem[2] = {0, 0};
  if (use_passes) {
    const int L = std::min(n, 5);  // low qubits always in the tile (coalesced runs)
    // Greedy cut of an op sequence into passes: a pass takes ops in order
    // while their targets fit in T tile qubits.
    auto build = [&](const std::vector<int>& order, bool reverse, std::vector<PassArg>& out) {
      std::set<int> S;
      std::vector<int> cur;
      auto reset_S = [&]() {
        S.clear();
        for (int q = 0; q < (T == n ? n : L); ++q) S.insert(q);
      };
      auto close_pass = [&]() {
        if (cur.empty()) { reset_S(); return; }
        for (int q = 0; (int)S.size() < T && q < n; ++q) S.insert(q);  // fill the tile to T qubits
        PassArg P;
        std::memset(&P, 0, sizeof(P));
        P.T = T;
        int k = 0, pos[64];
        for (int q : S) { P.S[k] = q; pos[q] = k; ++k; }
        P.gb = (int)gates.size();
        for (int i : cur) {
          const qs_op& o = ops[i];
          AdjGate G;
          std::memset(&G, 0, sizeof(G));
          G.slot = -1;
          if (is_1q_kind(o.kind)) {
            G.kind = AG_1Q;
            G.p0 = pos[o.q[0]];
            G.mat = i;
            if (reverse && o.param >= 0) {
              G.gkind = o.kind == QS_OP_RX ? 1 : o.kind == QS_OP_RY ? 2 : 3;
              G.slot = (int)param_of.size();
              param_of.push_back(o.param);
            }
          } else if (o.kind == QS_OP_MCX) {
            G.kind = AG_MCX;
            G.p0 = pos[o.q[o.nq - 1]];
            for (int c = 0; c + 1 < o.nq; ++c) G.cmask |= 1ull << o.q[c];
          } else if (o.kind == QS_OP_MCPHASE) {
            G.kind = AG_PHASE;
            for (int c = 0; c < o.nq; ++c) G.cmask |= 1ull << o.q[c];
            G.neg = (o.m[0] == -1.0 && o.m[1] == 0.0) ? 1 : 0;
            G.ph = make_float2((float)o.m[0], (float)-o.m[1]);
          } else {
            G.kind = AG_U2;
            G.p0 = pos[o.q[0]];
            G.p1 = pos[o.q[1]];
            G.mat = (int)u2s.size();
            Mat4 U;  // U^dag; the forward kernel transposes it back
            for (int r = 0; r < 4; ++r)
              for (int c = 0; c < 4; ++c)
                U.g[4 * r + c] = make_float2((float)o.m[2 * (4 * c + r)], (float)-o.m[2 * (4 * c + r) + 1]);
            u2s.push_back(U);
          }
          gates.push_back(G);
        }
        P.ge = (int)gates.size();
        out.push_back(P);
        cur.clear();
        reset_S();
      };
      // List scheduling: an op is ready when it is the next op of the order
      // on every qubit it touches (ops on disjoint qubits commute, and so do
      // their contributions to the gradient); a pass keeps taking ready ops
      // whose targets are in its tile, and adds the targets of the earliest
      // ready op to the tile while room is left.
      const int m = (int)order.size();
      std::vector<std::vector<int>> touch(m), targ(m);
      std::vector<std::vector<int>> per_q(n);  // positions in `order` touching each qubit
      for (int k = 0; k < m; ++k) {
        const qs_op& o = ops[order[k]];
        if (is_1q_kind(o.kind)) targ[k] = {o.q[0]};
        else if (o.kind == QS_OP_MCX) targ[k] = {o.q[o.nq - 1]};
        else if (o.kind == QS_OP_U2) targ[k] = {o.q[0], o.q[1]};
        touch[k].assign(o.q, o.q + o.nq);
        for (int q : touch[k]) per_q[q].push_back(k);
      }
      std::vector<size_t> head(n, 0);  // next unscheduled position per qubit
      std::vector<char> done(m, 0);
      auto ready = [&](int k) {
        for (int q : touch[k])
          if (per_q[q][head[q]] != k) return false;
        return true;
      };
      auto fits = [&](int k) {
        for (int q : targ[k])
          if (!S.count(q)) return false;
        return true;
      };
      int remaining = m, first = 0;
      reset_S();
      while (remaining > 0) {
        bool progress = true;
        while (progress) {
          progress = false;
          for (int k = first; k < m; ++k) {
            if (done[k] || !ready(k) || !fits(k)) continue;
            done[k] = 1;
            --remaining;
            for (int q : touch[k]) ++head[q];
            cur.push_back(order[k]);
            progress = true;
          }
          while (first < m && done[first]) ++first;
        }
        if (remaining == 0) break;
        // widen the tile with the earliest ready op's targets, or close the pass
        int pick = -1;
        for (int k = first; k < m && pick < 0; ++k)
          if (!done[k] && ready(k)) pick = k;
        std::set<int> need = S;
        need.insert(targ[pick].begin(), targ[pick].end());
        if ((int)need.size() <= T) {
          S = need;
        } else {
          close_pass();
        }
      }
      close_pass();
    };
    std::vector<int> order(nops);
    for (int i = 0; i < nops; ++i) order[i] = i;
    build(order, false, fpasses);
    std::reverse(order.begin(), order.end());
    build(order, true, rpasses);
    if (!fpasses.empty()) fpasses[0].from_zero = 1;
    const int nslots = (int)param_of.size();
    for (auto& P : rpasses) P.nslots = nslots;
    // device: gates | U2 matrices | slot -> parameter | partials
    const size_t gbytes = gates.size() * sizeof(AdjGate), ubytes = u2s.size() * sizeof(Mat4);
    const size_t pbytes = sizeof(int32_t) * std::max(nslots, 1);
    const size_t parts = (size_t)nb * std::max(nslots, 1) * ntiles;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    QS_CUDA(cudaMallocAsync(&pbuf, al(gbytes) + al(ubytes) + al(pbytes) + sizeof(double) * parts, h->stream));
    char* pc = static_cast<char*>(pbuf);
    d_gates = reinterpret_cast<AdjGate*>(pc);
    d_u2 = reinterpret_cast<Mat4*>(pc + al(gbytes));
    d_param_of = reinterpret_cast<int32_t*>(pc + al(gbytes) + al(ubytes));
    d_parts = reinterpret_cast<double*>(pc + al(gbytes) + al(ubytes) + al(pbytes));
    if (gbytes) QS_CUDA(cudaMemcpyAsync(d_gates, gates.data(), gbytes, cudaMemcpyHostToDevice, h->stream));
    if (ubytes) QS_CUDA(cudaMemcpyAsync(d_u2, u2s.data(), ubytes, cudaMemcpyHostToDevice, h->stream));
    if (nslots)
      QS_CUDA(cudaMemcpyAsync(d_param_of, param_of.data(), pbytes, cudaMemcpyHostToDevice, h->stream));
    pass_smem[0] = sizeof(float2) * ((size_t)1 << T) + 2 * 128 * sizeof(uint64_t);  // forward
    pass_smem[1] = sizeof(float2) * 2 * ((size_t)1 << T) + 2 * 128 * sizeof(uint64_t);
    QS_CUDA(cudaFuncSetAttribute(k_adj_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem[0]));
    QS_CUDA(cudaFuncSetAttribute(k_adj_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem[1]));
  }

  // ---- forward
  if (use_passes) {
    for (const PassArg& P : fpasses) {
      k_adj_pass<true><<<dim3((unsigned)ntiles, nb), kThreads, pass_smem[0], h->stream>>>(
          (float2*)work, vstride, P, d_gates, d_udag, nb, d_u2, nullptr);
      qs_after_launch(h, "k_adj_pass");
    }
  } else {
    // one circuit per vector, params substituted, through the batch planner
    std::vector<qs_op> all((size_t)nops * nb);
    std::vector<int64_t> ooff(nb + 1), soff(nb);
    std::vector<int32_t> widths(nb, n);
    for (int b = 0; b < nb; ++b) {
      ooff[b] = (int64_t)b * nops;
      soff[b] = (int64_t)(b * vstride);
      for (int i = 0; i < nops; ++i) {
        qs_op o = ops[i];
        if (o.param >= 0) o.m[0] = params[(size_t)b * nparams + o.param];
        all[(size_t)b * nops + i] = o;
      }
    }
    ooff[nb] = (int64_t)nops * nb;
    int rc = qs_batch_plan_create(h, nb, widths.data(), ooff.data(), all.data(), soff.data(), &fwd);
    if (rc != QS_OK) throw qs_error(rc, h->err);
    rc = qs_batch_plan_execute(h, fwd, work);
    if (rc != QS_OK) throw qs_error(rc, h->err);
  }

  // ---- lam = H psi, E = Re<psi|lam>
  TermL* dT = (TermL*)qs_upload_terms(h, 0, n, xm, zm, coefs, nterms);
  {
    dim3 grid((unsigned)std::min<uint64_t>((N + kThreads - 1) / kThreads, 64), nb);
    k_adj_hpsi<<<grid, kThreads, sizeof(TermL) * nterms, h->stream>>>((float2*)work, vstride, N, dT, nterms);
    qs_after_launch(h, "k_adj_hpsi");
    k_adj_dot<<<dim3(sd.nbx, nb), kThreads, 0, h->stream>>>((const float2*)work, vstride, N, sd.per, d_part);
    qs_after_launch(h, "k_adj_dot");
    k_adj_final<<<nb, kThreads, 0, h->stream>>>(d_part, sd.nbx, d_energy, 1, 0, 0);
    qs_after_launch(h, "k_adj_final");
  }

  // ---- reverse sweep
  if (use_passes) {
    for (const PassArg& P : rpasses) {
      k_adj_pass<false><<<dim3((unsigned)ntiles, nb), kThreads, pass_smem[1], h->stream>>>(
          (float2*)work, vstride, P, d_gates, d_udag, nb, d_u2, d_parts);
      qs_after_launch(h, "k_adj_pass");
    }
    if (!param_of.empty()) {
      k_adj_slots<<<nb, kThreads, 0, h->stream>>>(d_parts, (int)param_of.size(), ntiles, d_param_of, d_grads,
                                                  nparams);
      qs_after_launch(h, "k_adj_slots");
    }
  } else
  for (int i = nops - 1; i >= 0; --i) {
    const qs_op& o = ops[i];
    if (is_1q_kind(o.kind)) {
      const int t = o.q[0];
      int gk = 0;
      if (o.param >= 0) gk = o.kind == QS_OP_RX ? 1 : o.kind == QS_OP_RY ? 2 : o.kind == QS_OP_RZ ? 3 : 0;
      QS_CHECK_ARG(o.param < 0 || gk != 0, "only RX/RY/RZ ops may carry a parameter");
      k_adj_1q<<<dim3(sl.nbx, nb), kThreads, 0, h->stream>>>((float2*)work, vstride, N / 2, t,
                                                              d_udag + (size_t)i * nb, gk, sl.per, d_part);
      qs_after_launch(h, "k_adj_1q");
      if (gk) {
        k_adj_final<<<nb, kThreads, 0, h->stream>>>(d_part, sl.nbx, d_grads, nparams, o.param, 1);
        qs_after_launch(h, "k_adj_final");
      }
    } else if (o.kind == QS_OP_MCX) {
      std::vector<int> all_q(o.q, o.q + o.nq);
      uint64_t cmask = 0;
      for (int k = 0; k + 1 < o.nq; ++k) cmask |= 1ull << o.q[k];
      const uint64_t items = N >> o.nq;
      dim3 grid((unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + kThreads - 1) / kThreads, 64)), nb);
      k_adj_mcx<<<grid, kThreads, 0, h->stream>>>((float2*)work, vstride, items, sortedq(all_q), cmask, o.q[o.nq - 1]);
      qs_after_launch(h, "k_adj_mcx");
    } else if (o.kind == QS_OP_MCPHASE) {
      std::vector<int> all_q(o.q, o.q + o.nq);
      uint64_t mask = 0;
      for (int k = 0; k < o.nq; ++k) mask |= 1ull << o.q[k];
      const uint64_t items = N >> o.nq;
      const bool neg = (o.m[0] == -1.0 && o.m[1] == 0.0);
      dim3 grid((unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + kThreads - 1) / kThreads, 64)), nb);
      k_adj_phase<<<grid, kThreads, 0, h->stream>>>((float2*)work, vstride, items, sortedq(all_q), mask,
                                                     make_float2((float)o.m[0], (float)-o.m[1]), neg ? 1 : 0);
      qs_after_launch(h, "k_adj_phase");
    } else if (o.kind == QS_OP_U2) {
      Mat4 U;
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
          U.g[4 * r + c] = make_float2((float)o.m[2 * (4 * c + r)], (float)-o.m[2 * (4 * c + r) + 1]);
      const uint64_t items = N >> 2;
      dim3 grid((unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + kThreads - 1) / kThreads, 64)), nb);
      k_adj_2q<<<grid, kThreads, 0, h->stream>>>((float2*)work, vstride, items, o.q[0], o.q[1], U);
      qs_after_launch(h, "k_adj_2q");
    } else {
      throw qs_error(QS_ERR_INVALID, "op kind not supported by the adjoint sweep");
    }
  }
  QS_CUDA(cudaMemcpyAsync(grads, d_grads, sizeof(double) * (size_t)nb * nparams, cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaMemcpyAsync(energies, d_energy, sizeof(double) * nb, cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaFreeAsync(dbuf, h->stream));
  dbuf = nullptr;
  if (pbuf) QS_CUDA(cudaFreeAsync(pbuf, h->stream));
  pbuf = nullptr;
  QS_CUDA(cudaStreamSynchronize(h->stream));
  qs_batch_plan_destroy(fwd);
  fwd = nullptr;
  return QS_OK;
  }
  catch (const qs_error& e) {
    h->err = e.what();
    cudaStreamSynchronize(h->stream);
    if (dbuf) cudaFreeAsync(dbuf, h->stream);
    if (pbuf) cudaFreeAsync(pbuf, h->stream);
    if (fwd) qs_batch_plan_destroy(fwd);
    return e.code;
  }
  catch (const std::exception& e) {
    h->err = e.what();
    cudaStreamSynchronize(h->stream);
    if (dbuf) cudaFreeAsync(dbuf, h->stream);
    if (pbuf) cudaFreeAsync(pbuf, h->stream);
    if (fwd) qs_batch_plan_destroy(fwd);
    return QS_ERR_INVALID;
  }
}
