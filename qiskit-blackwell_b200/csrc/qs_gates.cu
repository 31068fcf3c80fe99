// qs_gates.cu — one-gate-per-launch kernels (the reference's per-op API).
//
// Every kernel streams the state in place with 64-bit indices and grid-stride
// loops sized to the SM count.  Wherever the touched amplitudes come in
// adjacent pairs the kernels use 128-bit accesses (two complex64 per float4).
// Dense gates use the compensated Dot2 evaluation (qs_common.cuh); diagonal
// gates the compensated Kahan complex product; X/CNOT/Toffoli/SWAP/Z/CZ are
// exact moves or negations.
#include "qs_api.h"
#include "qs_common.cuh"
#include <algorithm>
#include <cstdlib>

using namespace qs;

namespace {

struct G2 { float2 g[4]; };
struct G4 { float2 g[16]; };
struct Sorted { int pos[12]; int k; };

constexpr int kThreads = 256;

// Every kernel here is launched with programmatic dependent launch
// (qs_launch_pdl) and begins with pdl_begin().

// ------------------------------------------------------------ init --------
__global__ void k_state_init(float4* __restrict__ s4, uint64_t nvec, uint64_t index) {
  pdl_begin();
  for (uint64_t i = gtid(); i < nvec; i += gstride()) {
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if ((index >> 1) == i) { if (index & 1) v.z = 1.f; else v.x = 1.f; }
    s4[i] = v;
  }
}

// states back to back, each of 2^n amplitudes: amplitude 0 of each is 1.
__global__ void k_state_init_batched(float4* __restrict__ s4, uint64_t nvec, int n) {
  pdl_begin();
  uint64_t mask = (1ull << n) - 1ull;
  for (uint64_t i = gtid(); i < nvec; i += gstride()) {
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (((2 * i) & mask) == 0) v.x = 1.f;
    s4[i] = v;
  }
}

// ------------------------------------------------------------- 1Q ---------
__device__ __forceinline__ void apply2(const G2& G, float2& a0, float2& a1) {
  float2 r0[2] = {G.g[0], G.g[1]}, r1[2] = {G.g[2], G.g[3]}, v[2] = {a0, a1};
  float2 n0 = cdot_comp<2>(r0, v);
  float2 n1 = cdot_comp<2>(r1, v);
  a0 = n0; a1 = n1;
}

// A gate given by value, or read by every thread from device memory when gd
// is not null (callers whose matrix lives in a device tensor, so that no
// host copy and no stream synchronisation is needed).
__device__ __forceinline__ G2 gate2(const G2& G, const float2* __restrict__ gd) {
  if (!gd) return G;
  G2 R;
#pragma unroll
  for (int i = 0; i < 4; ++i) R.g[i] = gd[i];
  return R;
}

// target 0: the pair is one float4.
__global__ void k_1q_t0(float2* __restrict__ s, uint64_t npairs, G2 G0, const float2* __restrict__ gd) {
  pdl_begin();
  const G2 G = gate2(G0, gd);
  for (uint64_t p = gtid(); p < npairs; p += gstride()) {
    float4 v = ld4(s + 2 * p);
    float2 a0 = lo2(v), a1 = hi2(v);
    apply2(G, a0, a1);
    st4(s + 2 * p, a0, a1);
  }
}

// target t >= 1: two neighbouring pairs per thread, two float4 accesses.
__global__ void k_1q_tn(float2* __restrict__ s, uint64_t nitems, int t, G2 G0, const float2* __restrict__ gd) {
  pdl_begin();
  const G2 G = gate2(G0, gd);
  const uint64_t st = 1ull << t;
  for (uint64_t it = gtid(); it < nitems; it += gstride()) {
    uint64_t i0 = insert_zero(2 * it, t);
    float4 v0 = ld4(s + i0), v1 = ld4(s + i0 + st);
    float2 a0 = lo2(v0), b0 = hi2(v0), a1 = lo2(v1), b1 = hi2(v1);
    apply2(G, a0, a1);
    apply2(G, b0, b1);
    st4(s + i0, a0, b0);
    st4(s + i0 + st, a1, b1);
  }
}

// K <= 12 single-qubit gates whose matrices and targets are device arrays,
// applied in one launch (the device-tensor form of apply_gates_fused: no host
// copy of the gates, no stream synchronisation).  Each CTA stages tiles of
// 2^T amplitudes (T = min(n, 12)) whose qubits are the gates' distinct
// targets and the lowest other qubits, applies the gates to the tile in
// shared memory as an FMA chain per output (each FMA rounds once; the
// single-gate kernels' compensated Dot2 costs four times the arithmetic),
// and writes the tile back.  Gates on different qubits commute, so the gates
// are applied in groups of up to four on distinct tile positions, each gate
// after every earlier gate on its own qubit: a thread holds the 2^G
// amplitudes that a group mixes in registers and applies the group's gates
// there, one shared-memory sweep and barrier per group instead of per gate
// (ten gates on qubits 0, 2, ..., 18: three sweeps).  A group takes at most
// one position below 5 when the tile has 10 or more qubits, which keeps a
// warp's shared-memory accesses within two-way bank conflicts.  A target
// outside [0, n) makes every CTA return before it writes (bit 16 of the
// status word).
constexpr int kFusedMax = 12;
constexpr int kFusedGroup = 2;
constexpr int kFusedThreads = 512;

// One sweep of a group of G gates over the tile: gate b of the group (matrix
// M[b], tile position pos[b]) acts on register bit b of each thread's 2^G
// amplitudes; srt = the group's positions ascending.
template <int G>
__device__ __forceinline__ void fused_group_sweep(float2* __restrict__ tile, uint32_t tsize, const int* gidx,
                                                  const int* srt_s, const G2* sg, const int* spos) {
  int pos[G], srt[G];
  G2 M[G];
#pragma unroll
  for (int b = 0; b < G; ++b) {
    pos[b] = spos[gidx[b]];
    M[b] = sg[gidx[b]];
    srt[b] = srt_s[b];
  }
  uint32_t off[1 << G];
#pragma unroll
  for (int c = 0; c < (1 << G); ++c) {
    uint32_t o = 0;
#pragma unroll
    for (int b = 0; b < G; ++b)
      if ((c >> b) & 1) o |= 1u << pos[b];
    off[c] = o;
  }
  const uint32_t nitems = tsize >> G;
  for (uint32_t j = threadIdx.x; j < nitems; j += blockDim.x) {
    uint32_t base = j;
#pragma unroll
    for (int b = 0; b < G; ++b) base = (uint32_t)insert_zero(base, srt[b]);
    float2 a[1 << G];
#pragma unroll
    for (int c = 0; c < (1 << G); ++c) a[c] = tile[base | off[c]];
#pragma unroll
    for (int b = 0; b < G; ++b) {
#pragma unroll
      for (int c = 0; c < (1 << G); ++c) {
        if ((c >> b) & 1) continue;
        const int c1 = c | (1 << b);
        const float2 x0 = a[c], x1 = a[c1];
        a[c] = cfma2(M[b].g[0], x0, M[b].g[1], x1);
        a[c1] = cfma2(M[b].g[2], x0, M[b].g[3], x1);
      }
    }
#pragma unroll
    for (int c = 0; c < (1 << G); ++c) tile[base | off[c]] = a[c];
  }
}
__global__ void __launch_bounds__(kFusedThreads, 2) k_fused1q_dev(float2* __restrict__ s, int n, const float2* __restrict__ gates,
                                                          const int32_t* __restrict__ targets, int K,
                                                          uint32_t* status) {
  pdl_begin();
  extern __shared__ float2 tile[];
  __shared__ G2 sg[kFusedMax];
  __shared__ int st[kFusedMax];     // targets
  __shared__ int spos[kFusedMax];   // tile position of gate k's target
  __shared__ int sq[kFusedMax];     // tile qubits, ascending
  __shared__ uint64_t dep[2][64];   // tile index bits -> state index bits (6 + 6)
  __shared__ int gidx[kFusedMax][kFusedGroup];  // groups: gate indices, application order
  __shared__ int gsrt[kFusedMax][kFusedGroup];  // groups: tile positions ascending
  __shared__ int gsize[kFusedMax];
  __shared__ int s_ngroups;
  __shared__ int s_ok;
  const int T = n < kFusedMax ? n : kFusedMax;
  // one round trip for the gates' matrices and targets, then thread 0 picks
  // the tile qubits from shared memory
  if ((int)threadIdx.x < K) st[threadIdx.x] = targets[threadIdx.x];
  if ((int)threadIdx.x < 4 * K) sg[threadIdx.x >> 2].g[threadIdx.x & 3] = gates[threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    // thread 0 alone, while the CTA waits at the barrier: the targets and
    // positions live in registers (loops unrolled over kFusedMax), so the
    // setup costs no shared-memory round trips
    int tg[kFusedMax];
    uint64_t m = 0;
    int ok = 1;
#pragma unroll
    for (int k = 0; k < kFusedMax; ++k) {
      tg[k] = k < K ? st[k] : 0;
      if (k < K) {
        if (tg[k] < 0 || tg[k] >= n) ok = 0; else m |= 1ull << tg[k];
      }
    }
    for (int q = 0; q < n && __popcll(m) < T; ++q) m |= 1ull << q;
    {
      uint64_t r = m;
      for (int j = 0; r != 0; ++j, r &= r - 1) sq[j] = __ffsll((long long)r) - 1;
    }
    if (ok) {
      int sp[kFusedMax];
      uint32_t same[kFusedMax];  // earlier gates on the same position
#pragma unroll
      for (int k = 0; k < kFusedMax; ++k) {
        sp[k] = __popcll(m & ((1ull << tg[k]) - 1ull));
        spos[k] = sp[k];
        same[k] = 0;
#pragma unroll
        for (int k2 = 0; k2 < k; ++k2)
          if (sp[k2] == sp[k]) same[k] |= 1u << k2;
      }
      // groups: scan the unscheduled gates in order and take gate k unless
      // an earlier unscheduled gate (in this group or later) has its
      // position, the group is full, or it would be a second low position
      const int lowlim = T >= 10 ? 5 : 0;
      const uint32_t all = (1u << K) - 1u;
      uint32_t done = 0;
      int ng = 0;
      while (done != all) {
        int cnt = 0;
        uint32_t used = 0, pick = 0;
        bool low = false;
#pragma unroll
        for (int k = 0; k < kFusedMax; ++k) {
          const int p = sp[k];
          if (k < K && cnt < kFusedGroup && !((done >> k) & 1u) && !(same[k] & ~done) && !(p < lowlim && low)) {
            gidx[ng][cnt++] = k;
            used |= 1u << p;
            pick |= 1u << k;
            if (p < lowlim) low = true;
          }
        }
        done |= pick;
        uint32_t r = used;
        for (int j = 0; r != 0; ++j, r &= r - 1) gsrt[ng][j] = __ffs((int)r) - 1;
        gsize[ng++] = cnt;
      }
      s_ngroups = ng;
    } else if (blockIdx.x == 0) {
      atomicOr(status, 16u);
    }
    s_ok = ok;
  }
  __syncthreads();
  if (!s_ok) return;
  for (int e = threadIdx.x; e < 128; e += blockDim.x) {
    const int part = e >> 6, x = e & 63;
    uint64_t d = 0;
    for (int b = 0; b < 6; ++b) {
      const int kk = 6 * part + b;
      if (kk < T && ((x >> b) & 1)) d |= 1ull << sq[kk];
    }
    dep[part][x] = d;
  }
  __syncthreads();
  const uint32_t tsize = 1u << T;
  const uint64_t ntiles = 1ull << (n - T);
  for (uint64_t tl = blockIdx.x; tl < ntiles; tl += gridDim.x) {
    uint64_t gbase = tl;
    for (int k = 0; k < T; ++k) gbase = insert_zero(gbase, sq[k]);
#pragma unroll 16
    for (uint32_t i = threadIdx.x; i < tsize; i += blockDim.x) tile[i] = s[gbase | dep[0][i & 63] | dep[1][i >> 6]];
    __syncthreads();
    for (int g = 0; g < s_ngroups; ++g) {
      switch (gsize[g]) {
        case 1: fused_group_sweep<1>(tile, tsize, gidx[g], gsrt[g], sg, spos); break;
        default: fused_group_sweep<2>(tile, tsize, gidx[g], gsrt[g], sg, spos); break;
      }
      __syncthreads();
    }
#pragma unroll 8
    for (uint32_t i = threadIdx.x; i < tsize; i += blockDim.x) s[gbase | dep[0][i & 63] | dep[1][i >> 6]] = tile[i];
    __syncthreads();
  }
}

// ------------------------------------------------------------- 2Q ---------
__device__ __forceinline__ void apply4(const G4& G, float2& a0, float2& a1, float2& a2, float2& a3) {
  float2 v[4] = {a0, a1, a2, a3};
  float2 o[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    float2 row[4] = {G.g[4 * r], G.g[4 * r + 1], G.g[4 * r + 2], G.g[4 * r + 3]};
    o[r] = cdot_comp<4>(row, v);
  }
  a0 = o[0]; a1 = o[1]; a2 = o[2]; a3 = o[3];
}

// As gate2 for 4x4; swap: exchange the roles of matrix index bits 0 and 1.
__device__ __forceinline__ G4 gate4(const G4& G, const float2* __restrict__ gd, int swap) {
  if (!gd) return G;
  G4 R;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int pr = swap ? ((r & 1) << 1 | r >> 1) : r, pc = swap ? ((c & 1) << 1 | c >> 1) : c;
      R.g[4 * r + c] = gd[4 * pr + pc];
    }
  return R;
}

// lo == 0: a00,a01 adjacent and a10,a11 adjacent.
__global__ void k_2q_lo0(float2* __restrict__ s, uint64_t nquads, int hi, G4 G0, const float2* __restrict__ gd,
                         int swap) {
  pdl_begin();
  const G4 G = gate4(G0, gd, swap);
  const uint64_t sh = 1ull << hi;
  for (uint64_t it = gtid(); it < nquads; it += gstride()) {
    uint64_t i00 = insert_zero(insert_zero(it, 0), hi);
    float4 v0 = ld4(s + i00), v1 = ld4(s + i00 + sh);
    float2 a0 = lo2(v0), a1 = hi2(v0), a2 = lo2(v1), a3 = hi2(v1);
    apply4(G, a0, a1, a2, a3);
    st4(s + i00, a0, a1);
    st4(s + i00 + sh, a2, a3);
  }
}

// lo >= 1: two neighbouring quads per thread.
__global__ void k_2q_gen(float2* __restrict__ s, uint64_t nitems, int lo, int hi, G4 G0,
                         const float2* __restrict__ gd, int swap) {
  pdl_begin();
  const G4 G = gate4(G0, gd, swap);
  const uint64_t sl = 1ull << lo, sh = 1ull << hi;
  for (uint64_t it = gtid(); it < nitems; it += gstride()) {
    uint64_t i00 = insert_zero(insert_zero(2 * it, lo), hi);
    float4 v00 = ld4(s + i00), v01 = ld4(s + i00 + sl), v10 = ld4(s + i00 + sh), v11 = ld4(s + i00 + sl + sh);
    float2 a0 = lo2(v00), a1 = lo2(v01), a2 = lo2(v10), a3 = lo2(v11);
    float2 b0 = hi2(v00), b1 = hi2(v01), b2 = hi2(v10), b3 = hi2(v11);
    apply4(G, a0, a1, a2, a3);
    apply4(G, b0, b1, b2, b3);
    st4(s + i00, a0, b0);
    st4(s + i00 + sl, a1, b1);
    st4(s + i00 + sh, a2, b2);
    st4(s + i00 + sl + sh, a3, b3);
  }
}

// ----------------------------------------------------------- diagonal -----
__global__ void k_diag1(float2* __restrict__ s, uint64_t nvec, int t, float2 d0v, float2 d1v,
                        const float2* __restrict__ gd) {
  pdl_begin();
  const float2 d0 = gd ? gd[0] : d0v, d1 = gd ? gd[1] : d1v;
  for (uint64_t i = gtid(); i < nvec; i += gstride()) {
    uint64_t idx = 2 * i;
    float4 v = ld4(s + idx);
    float2 e0, e1;
    if (t == 0) { e0 = d0; e1 = d1; }
    else { e0 = e1 = ((idx >> t) & 1) ? d1 : d0; }
    st4(s + idx, cmul_comp(lo2(v), e0), cmul_comp(hi2(v), e1));
  }
}

// Only amplitudes with bit t = 1 (half the traffic).
__global__ void k_phase_t0(float2* __restrict__ s, uint64_t npairs, float2 ph) {
  pdl_begin();
  for (uint64_t p = gtid(); p < npairs; p += gstride()) {
    uint64_t idx = 2 * p + 1;
    s[idx] = cmul_comp(s[idx], ph);
  }
}
__global__ void k_phase_tn(float2* __restrict__ s, uint64_t nitems, int t, float2 ph) {
  pdl_begin();
  for (uint64_t it = gtid(); it < nitems; it += gstride()) {
    uint64_t idx = insert_zero(2 * it, t) | (1ull << t);
    float4 v = ld4(s + idx);
    st4(s + idx, cmul_comp(lo2(v), ph), cmul_comp(hi2(v), ph));
  }
}

__global__ void k_diag2(float2* __restrict__ s, uint64_t nvec, int q0, int q1, G2 D0, const float2* __restrict__ gd) {
  pdl_begin();
  const G2 D = gate2(D0, gd);
  for (uint64_t i = gtid(); i < nvec; i += gstride()) {
    uint64_t idx = 2 * i;
    float4 v = ld4(s + idx);
    uint64_t j = idx + 1;
    int s0 = (int)(((idx >> q1) & 1) << 1 | ((idx >> q0) & 1));
    int s1 = (int)(((j >> q1) & 1) << 1 | ((j >> q0) & 1));
    st4(s + idx, cmul_comp(lo2(v), D.g[s0]), cmul_comp(hi2(v), D.g[s1]));
  }
}

// ------------------------------------------------- multi-controlled -------
__global__ void k_mc1q(float2* __restrict__ s, uint64_t nitems, Sorted P, uint64_t cmask, int t, G2 G0,
                       const float2* __restrict__ gd) {
  pdl_begin();
  const G2 G = gate2(G0, gd);
  const uint64_t st = 1ull << t;
  for (uint64_t it = gtid(); it < nitems; it += gstride()) {
    uint64_t i0 = insert_zeros(it, P.pos, P.k) | cmask;
    float2 a0 = s[i0], a1 = s[i0 | st];
    apply2(G, a0, a1);
    s[i0] = a0;
    s[i0 | st] = a1;
  }
}

__global__ void k_mc2q(float2* __restrict__ s, uint64_t nitems, Sorted P, uint64_t cmask, int lo, int hi, G4 G0,
                       const float2* __restrict__ gd) {
  pdl_begin();
  const G4 G = gate4(G0, gd, 0);
  const uint64_t sl = 1ull << lo, sh = 1ull << hi;
  for (uint64_t it = gtid(); it < nitems; it += gstride()) {
    uint64_t i = insert_zeros(it, P.pos, P.k) | cmask;
    float2 a0 = s[i], a1 = s[i | sl], a2 = s[i | sh], a3 = s[i | sl | sh];
    apply4(G, a0, a1, a2, a3);
    s[i] = a0; s[i | sl] = a1; s[i | sh] = a2; s[i | sl | sh] = a3;
  }
}

// ---------------------------------------------------------- exact ---------
__global__ void k_x_t0(float2* __restrict__ s, uint64_t npairs) {
  pdl_begin();
  for (uint64_t p = gtid(); p < npairs; p += gstride()) {
    float4 v = ld4(s + 2 * p);
    st4(s + 2 * p, hi2(v), lo2(v));
  }
}
__global__ void k_x_tn(float2* __restrict__ s, uint64_t nitems, int t) {
  pdl_begin();
  const uint64_t st = 1ull << t;
  for (uint64_t it = gtid(); it < nitems; it += gstride()) {
    uint64_t i0 = insert_zero(2 * it, t);
    float4 v0 = ld4(s + i0), v1 = ld4(s + i0 + st);
    *reinterpret_cast<float4*>(s + i0) = v1;
    *reinterpret_cast<float4*>(s + i0 + st) = v0;
  }
}
__global__ void k_mcx(float2* __restrict__ s, uint64_t nitems, Sorted P, uint64_t cmask, int t) {
  pdl_begin();
  const uint64_t st = 1ull << t;
  for (uint64_t it = gtid(); it < nitems; it += gstride()) {
    uint64_t i0 = insert_zeros(it, P.pos, P.k) | cmask;
    float2 a0 = s[i0], a1 = s[i0 | st];
    s[i0] = a1;
    s[i0 | st] = a0;
  }
}
__global__ void k_mcswap(float2* __restrict__ s, uint64_t nitems, Sorted P, uint64_t cmask, int t0, int t1) {
  pdl_begin();
  const uint64_t s0 = 1ull << t0, s1 = 1ull << t1;
  for (uint64_t it = gtid(); it < nitems; it += gstride()) {
    uint64_t i = insert_zeros(it, P.pos, P.k) | cmask;
    float2 a = s[i | s0], b = s[i | s1];
    s[i | s0] = b;
    s[i | s1] = a;
  }
}
__global__ void k_mcz(float2* __restrict__ s, uint64_t nitems, Sorted P, uint64_t mask) {
  pdl_begin();
  for (uint64_t it = gtid(); it < nitems; it += gstride()) {
    uint64_t i = insert_zeros(it, P.pos, P.k) | mask;
    float2 a = s[i];
    s[i] = make_float2(-a.x, -a.y);
  }
}

// --------------------------------------------------------- host side ------
inline float2 f2(const float* p) { return make_float2(p[0], p[1]); }

G2 load_g2(const float* g) {
  QS_CHECK_ARG(g != nullptr, "gate pointer is null");
  G2 G;
  for (int i = 0; i < 4; ++i) G.g[i] = f2(g + 2 * i);
  return G;
}

G4 load_g4(const float* g) {
  QS_CHECK_ARG(g != nullptr, "gate pointer is null");
  G4 G;
  for (int i = 0; i < 16; ++i) G.g[i] = f2(g + 2 * i);
  return G;
}

// Swap the roles of matrix index bits 0 and 1 (basis order 00,01,10,11).
G4 swap_bits(const G4& G) {
  static const int perm[4] = {0, 2, 1, 3};
  G4 R;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) R.g[4 * r + c] = G.g[4 * perm[r] + perm[c]];
  return R;
}

Sorted make_sorted(const int* qs, int k) {
  QS_CHECK_ARG(k <= 12, "too many qubits in a controlled gate");
  Sorted P;
  for (int i = 0; i < k; ++i) P.pos[i] = qs[i];
  std::sort(P.pos, P.pos + k);
  for (int i = 1; i < k; ++i) QS_CHECK_ARG(P.pos[i] != P.pos[i - 1], "duplicate qubit in gate");
  for (int i = k; i < 12; ++i) P.pos[i] = 0;
  P.k = k;
  return P;
}

void check_controls(const int* controls, int nc, int n) {
  QS_CHECK_ARG(nc >= 0 && nc <= QS_MAX_CONTROLS, "controls must have 0-7 elements");
  QS_CHECK_ARG(nc == 0 || controls != nullptr, "controls pointer is null");
  for (int i = 0; i < nc; ++i) qs_check_qubit(controls[i], n, "control");
}

#define LAUNCH(h, kern, items, ...)                                              \
  do {                                                                          \
    uint64_t _items = (items);                                                  \
    if (_items) {                                                               \
      qs_launch_pdl(h, kern, dim3((unsigned)qs_blocks_for(h, _items, kThreads)), dim3(kThreads), 0, __VA_ARGS__); \
      qs_after_launch(h, #kern);                                                \
    }                                                                           \
  } while (0)

}  // namespace

// Exposed to other units (apply_gates_fused fallback and tests).
void qs_launch_1q(qs_context* h, float2* s, uint64_t npairs_total, int t, const G2& G,
                  const float2* gd = nullptr);

void qs_launch_1q(qs_context* h, float2* s, uint64_t npairs, int t, const G2& G, const float2* gd) {
  if (t == 0) LAUNCH(h, k_1q_t0, npairs, s, npairs, G, gd);
  else LAUNCH(h, k_1q_tn, npairs / 2, s, npairs / 2, t, G, gd);
}

extern "C" {

int qs_state_init(qs_handle_t h, void* state, int n) {
  return qs_state_init_basis(h, state, n, 0);
}

int qs_state_init_basis(qs_handle_t h, void* state, int n, uint64_t index) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(index < (1ull << n), "basis index out of range");
  uint64_t nvec = (1ull << n) / 2;
  LAUNCH(h, k_state_init, nvec, (float4*)state, nvec, index);
  QS_API_END(h)
}

int qs_state_alloc(qs_handle_t h, int n, void** out) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(out != nullptr, "out is null");
  *out = nullptr;
  QS_CHECK_ARG(n >= 1 && n <= QS_MAX_QUBITS, "n_qubits out of range [1, 34]");
  void* p = nullptr;
  const cudaError_t e = cudaMallocAsync(&p, (size_t)8 << n, h->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw qs_error(QS_ERR_NOMEM, std::string("state allocation: ") + cudaGetErrorString(e));
  }
  *out = p;
  QS_API_END(h)
}

int qs_state_free(qs_handle_t h, void* state) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  if (state) QS_CUDA(cudaFreeAsync(state, h->stream));
  QS_API_END(h)
}

int qs_state_copy_to_host(qs_handle_t h, const void* state, int n, void* host) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(host != nullptr, "host buffer is null");
  QS_CUDA(cudaMemcpyAsync(host, state, (size_t)8 << n, cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaStreamSynchronize(h->stream));
  QS_API_END(h)
}

int qs_state_copy_from_host(qs_handle_t h, void* state, int n, const void* host) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(host != nullptr, "host buffer is null");
  QS_CUDA(cudaMemcpyAsync(state, host, (size_t)8 << n, cudaMemcpyHostToDevice, h->stream));
  QS_CUDA(cudaStreamSynchronize(h->stream));
  QS_API_END(h)
}

int qs_state_init_batched(qs_handle_t h, void* states, int n_states, int n) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(states, n);
  QS_CHECK_ARG(n_states >= 0, "n_states must be >= 0");
  uint64_t nvec = (uint64_t)n_states * ((1ull << n) / 2);
  LAUNCH(h, k_state_init_batched, nvec, (float4*)states, nvec, n);
  QS_API_END(h)
}

int qs_apply_1q(qs_handle_t h, void* state, int n, const float* gate, int t) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t, n, "target");
  G2 G = load_g2(gate);
  qs_launch_1q(h, (float2*)state, 1ull << (n - 1), t, G);
  QS_API_END(h)
}

int qs_apply_1q_batched(qs_handle_t h, void* states, int n_states, int n, const float* gate, int t) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(states, n);
  qs_check_qubit(t, n, "target");
  QS_CHECK_ARG(n_states >= 0, "n_states must be >= 0");
  G2 G = load_g2(gate);
  // Pair index p ranges over n_states * 2^(n-1); inserting a zero at t < n
  // leaves the state index in the bits above n.
  qs_launch_1q(h, (float2*)states, (uint64_t)n_states << (n - 1), t, G);
  QS_API_END(h)
}

// Gates whose matrix is a device array (complex64, row-major): the kernel
// reads it, so the call neither copies it to the host nor waits for the
// stream.  The pointer must be device memory of the handle's own GPU (or
// managed memory): a gate on another GPU would be read across the link, or
// fault when peer access is off.
// The last four pointers that passed are remembered per handle together with
// the device each was checked for (gate tensors are usually reused call after
// call).  An address that was freed and handed out again by another
// allocation of the same GPU is still device memory of that GPU, so the
// remembered answer stays true for it.
static void check_dev_ptr(qs_context* h, const void* p, const char* what) {
  QS_CHECK_ARG(p != nullptr && ((uintptr_t)p & 7u) == 0, std::string(what) + " must be 8-byte aligned");
  for (int k = 0; k < 4; ++k)
    if (p == h->dev_ptr_ok[k] && h->dev_ptr_ok_device[k] == h->device) return;
  cudaPointerAttributes a;
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) (void)cudaGetLastError();  // clear the sticky-free error state of the query
  QS_CHECK_ARG(e == cudaSuccess && (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged),
               std::string(what) + " is not device memory");
  QS_CHECK_ARG(a.type == cudaMemoryTypeManaged || a.device == h->device,
               std::string(what) + " is device memory of GPU " + std::to_string(a.device) +
                   ", not of the handle's GPU " + std::to_string(h->device));
  h->dev_ptr_ok[h->dev_ptr_next] = p;
  h->dev_ptr_ok_device[h->dev_ptr_next] = h->device;
  h->dev_ptr_next = (h->dev_ptr_next + 1) & 3;
}

int qs_apply_1q_dev(qs_handle_t h, void* state, int n, const void* gate_dev, int t) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t, n, "target");
  check_dev_ptr(h, gate_dev, "gate");
  qs_launch_1q(h, (float2*)state, 1ull << (n - 1), t, G2{}, static_cast<const float2*>(gate_dev));
  QS_API_END(h)
}

int qs_apply_gates_fused_dev(qs_handle_t h, void* state, int n, const void* gates_dev, const void* targets_dev,
                             int n_gates) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(n_gates >= 0, "n_gates must be >= 0");
  if (n_gates == 0) return QS_OK;
  check_dev_ptr(h, gates_dev, "gates");
  QS_CHECK_ARG(((uintptr_t)targets_dev & 3u) == 0, "targets must be 4-byte aligned");
  check_dev_ptr(h, targets_dev, "targets");
  const int T = std::min(n, kFusedMax);
  const size_t smem = sizeof(float2) << T;
  const uint64_t ntiles = 1ull << (n - T);
  const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)h->sm_count * 6);
  const float2* g = static_cast<const float2*>(gates_dev);
  const int32_t* t = static_cast<const int32_t*>(targets_dev);
  // at most 12 gates per launch, so their distinct targets always fit a tile
  for (int k0 = 0; k0 < n_gates; k0 += kFusedMax) {
    const int K = std::min(kFusedMax, n_gates - k0);
    k_fused1q_dev<<<grid, kFusedThreads, smem, h->stream>>>((float2*)state, n, g + 4 * k0, t + k0, K, h->dev_status);
    qs_after_launch(h, "k_fused1q_dev");
  }
  QS_API_END(h)
}

int qs_apply_2q_dev(qs_handle_t h, void* state, int n, const void* gate_dev, int q0, int q1) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(n >= 2, "a 2-qubit gate needs n >= 2");
  qs_check_qubit(q0, n, "qubit0");
  qs_check_qubit(q1, n, "qubit1");
  QS_CHECK_ARG(q0 != q1, "qubit0 and qubit1 must differ");
  check_dev_ptr(h, gate_dev, "gate");
  const int lo = std::min(q0, q1), hi = std::max(q0, q1), swap = q0 > q1 ? 1 : 0;
  const float2* gd = static_cast<const float2*>(gate_dev);
  uint64_t nquads = 1ull << (n - 2);
  if (lo == 0) LAUNCH(h, k_2q_lo0, nquads, (float2*)state, nquads, hi, G4{}, gd, swap);
  else LAUNCH(h, k_2q_gen, nquads / 2, (float2*)state, nquads / 2, lo, hi, G4{}, gd, swap);
  QS_API_END(h)
}

int qs_apply_diag1_dev(qs_handle_t h, void* state, int n, const void* diag_dev, int t) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t, n, "target");
  check_dev_ptr(h, diag_dev, "diag");
  uint64_t nvec = (1ull << n) / 2;
  LAUNCH(h, k_diag1, nvec, (float2*)state, nvec, t, make_float2(0.f, 0.f), make_float2(0.f, 0.f),
         static_cast<const float2*>(diag_dev));
  QS_API_END(h)
}

int qs_apply_mc1q_dev(qs_handle_t h, void* state, int n, const void* gate_dev, const int* controls, int nc, int t) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t, n, "target");
  check_controls(controls, nc, n);
  check_dev_ptr(h, gate_dev, "gate");
  const float2* gd = static_cast<const float2*>(gate_dev);
  if (nc == 0) { qs_launch_1q(h, (float2*)state, 1ull << (n - 1), t, G2{}, gd); return QS_OK; }
  int all[QS_MAX_CONTROLS + 1];
  uint64_t cmask = 0;
  for (int i = 0; i < nc; ++i) {
    QS_CHECK_ARG(controls[i] != t, "target_qubit must not appear in controls");
    all[i] = controls[i];
    cmask |= 1ull << controls[i];
  }
  all[nc] = t;
  Sorted P = make_sorted(all, nc + 1);
  QS_CHECK_ARG(nc + 1 <= n, "more gate qubits than state qubits");
  uint64_t items = 1ull << (n - nc - 1);
  LAUNCH(h, k_mc1q, items, (float2*)state, items, P, cmask, t, G2{}, gd);
  QS_API_END(h)
}

int qs_apply_2q(qs_handle_t h, void* state, int n, const float* gate, int q0, int q1) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(n >= 2, "a 2-qubit gate needs n >= 2");
  qs_check_qubit(q0, n, "qubit0");
  qs_check_qubit(q1, n, "qubit1");
  QS_CHECK_ARG(q0 != q1, "qubit0 and qubit1 must differ");
  G4 G = load_g4(gate);
  int lo = q0, hi = q1;
  if (q0 > q1) { G = swap_bits(G); lo = q1; hi = q0; }
  uint64_t nquads = 1ull << (n - 2);
  if (lo == 0) LAUNCH(h, k_2q_lo0, nquads, (float2*)state, nquads, hi, G, nullptr, 0);
  else LAUNCH(h, k_2q_gen, nquads / 2, (float2*)state, nquads / 2, lo, hi, G, nullptr, 0);
  QS_API_END(h)
}

int qs_apply_diag1(qs_handle_t h, void* state, int n, const float* diag, int t) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t, n, "target");
  QS_CHECK_ARG(diag != nullptr, "diag pointer is null");
  uint64_t nvec = (1ull << n) / 2;
  LAUNCH(h, k_diag1, nvec, (float2*)state, nvec, t, f2(diag), f2(diag + 2), nullptr);
  QS_API_END(h)
}

int qs_apply_phase(qs_handle_t h, void* state, int n, float re, float im, int t) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t, n, "target");
  float2 ph = make_float2(re, im);
  uint64_t npairs = 1ull << (n - 1);
  if (t == 0) LAUNCH(h, k_phase_t0, npairs, (float2*)state, npairs, ph);
  else LAUNCH(h, k_phase_tn, npairs / 2, (float2*)state, npairs / 2, t, ph);
  QS_API_END(h)
}

int qs_apply_diag2(qs_handle_t h, void* state, int n, const float* diag, int q0, int q1) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(n >= 2, "a 2-qubit gate needs n >= 2");
  qs_check_qubit(q0, n, "qubit0");
  qs_check_qubit(q1, n, "qubit1");
  QS_CHECK_ARG(q0 != q1, "qubit0 and qubit1 must differ");
  QS_CHECK_ARG(diag != nullptr, "diag pointer is null");
  G2 D = load_g2(diag);
  int lo = std::min(q0, q1), hi = std::max(q0, q1);
  uint64_t nvec = (1ull << n) / 2;
  LAUNCH(h, k_diag2, nvec, (float2*)state, nvec, lo, hi, D, nullptr);
  QS_API_END(h)
}

int qs_apply_diag2_dev(qs_handle_t h, void* state, int n, const void* diag_dev, int q0, int q1) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(n >= 2, "a 2-qubit gate needs n >= 2");
  qs_check_qubit(q0, n, "qubit0");
  qs_check_qubit(q1, n, "qubit1");
  QS_CHECK_ARG(q0 != q1, "qubit0 and qubit1 must differ");
  check_dev_ptr(h, diag_dev, "diag");
  const int lo = std::min(q0, q1), hi = std::max(q0, q1);
  const uint64_t nvec = (1ull << n) / 2;
  LAUNCH(h, k_diag2, nvec, (float2*)state, nvec, lo, hi, G2{}, static_cast<const float2*>(diag_dev));
  QS_API_END(h)
}

int qs_apply_mc1q(qs_handle_t h, void* state, int n, const float* gate, const int* controls, int nc, int t) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t, n, "target");
  check_controls(controls, nc, n);
  G2 G = load_g2(gate);
  if (nc == 0) { qs_launch_1q(h, (float2*)state, 1ull << (n - 1), t, G); return QS_OK; }
  int all[QS_MAX_CONTROLS + 1];
  uint64_t cmask = 0;
  for (int i = 0; i < nc; ++i) {
    QS_CHECK_ARG(controls[i] != t, "target_qubit must not appear in controls");
    all[i] = controls[i];
    cmask |= 1ull << controls[i];
  }
  all[nc] = t;
  Sorted P = make_sorted(all, nc + 1);
  QS_CHECK_ARG(nc + 1 <= n, "more gate qubits than state qubits");
  uint64_t items = 1ull << (n - nc - 1);
  LAUNCH(h, k_mc1q, items, (float2*)state, items, P, cmask, t, G, nullptr);
  QS_API_END(h)
}

int qs_apply_mc2q(qs_handle_t h, void* state, int n, const float* gate, const int* controls, int nc, int t0, int t1) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t0, n, "target0");
  qs_check_qubit(t1, n, "target1");
  QS_CHECK_ARG(t0 != t1, "target0 and target1 must differ");
  check_controls(controls, nc, n);
  QS_CHECK_ARG(nc + 2 <= n, "more gate qubits than state qubits");
  G4 G = load_g4(gate);
  int lo = std::min(t0, t1), hi = std::max(t0, t1);
  int all[QS_MAX_CONTROLS + 2];
  uint64_t cmask = 0;
  for (int i = 0; i < nc; ++i) {
    QS_CHECK_ARG(controls[i] != t0 && controls[i] != t1, "target qubits must not appear in controls");
    all[i] = controls[i];
    cmask |= 1ull << controls[i];
  }
  all[nc] = lo;
  all[nc + 1] = hi;
  Sorted P = make_sorted(all, nc + 2);
  uint64_t items = 1ull << (n - nc - 2);
  LAUNCH(h, k_mc2q, items, (float2*)state, items, P, cmask, lo, hi, G, nullptr);
  QS_API_END(h)
}

int qs_apply_mc2q_dev(qs_handle_t h, void* state, int n, const void* gate_dev, const int* controls, int nc, int t0,
                      int t1) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t0, n, "target0");
  qs_check_qubit(t1, n, "target1");
  QS_CHECK_ARG(t0 != t1, "target0 and target1 must differ");
  check_controls(controls, nc, n);
  QS_CHECK_ARG(nc + 2 <= n, "more gate qubits than state qubits");
  check_dev_ptr(h, gate_dev, "gate");
  const int lo = std::min(t0, t1), hi = std::max(t0, t1);
  int all[QS_MAX_CONTROLS + 2];
  uint64_t cmask = 0;
  for (int i = 0; i < nc; ++i) {
    QS_CHECK_ARG(controls[i] != t0 && controls[i] != t1, "target qubits must not appear in controls");
    all[i] = controls[i];
    cmask |= 1ull << controls[i];
  }
  all[nc] = lo;
  all[nc + 1] = hi;
  Sorted P = make_sorted(all, nc + 2);
  const uint64_t items = 1ull << (n - nc - 2);
  LAUNCH(h, k_mc2q, items, (float2*)state, items, P, cmask, lo, hi, G4{}, static_cast<const float2*>(gate_dev));
  QS_API_END(h)
}

int qs_apply_mcx(qs_handle_t h, void* state, int n, const int* controls, int nc, int t) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t, n, "target");
  check_controls(controls, nc, n);
  QS_CHECK_ARG(nc + 1 <= n, "more gate qubits than state qubits");
  if (nc == 0) {
    uint64_t npairs = 1ull << (n - 1);
    if (t == 0) LAUNCH(h, k_x_t0, npairs, (float2*)state, npairs);
    else LAUNCH(h, k_x_tn, npairs / 2, (float2*)state, npairs / 2, t);
    return QS_OK;
  }
  int all[QS_MAX_CONTROLS + 1];
  uint64_t cmask = 0;
  for (int i = 0; i < nc; ++i) {
    QS_CHECK_ARG(controls[i] != t, "target_qubit must not appear in controls");
    all[i] = controls[i];
    cmask |= 1ull << controls[i];
  }
  all[nc] = t;
  Sorted P = make_sorted(all, nc + 1);
  uint64_t items = 1ull << (n - nc - 1);
  LAUNCH(h, k_mcx, items, (float2*)state, items, P, cmask, t);
  QS_API_END(h)
}

int qs_apply_mcswap(qs_handle_t h, void* state, int n, const int* controls, int nc, int t0, int t1) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t0, n, "target0");
  qs_check_qubit(t1, n, "target1");
  QS_CHECK_ARG(t0 != t1, "target0 and target1 must differ");
  check_controls(controls, nc, n);
  QS_CHECK_ARG(nc + 2 <= n, "more gate qubits than state qubits");
  int all[QS_MAX_CONTROLS + 2];
  uint64_t cmask = 0;
  for (int i = 0; i < nc; ++i) {
    QS_CHECK_ARG(controls[i] != t0 && controls[i] != t1, "target qubits must not appear in controls");
    all[i] = controls[i];
    cmask |= 1ull << controls[i];
  }
  all[nc] = t0;
  all[nc + 1] = t1;
  Sorted P = make_sorted(all, nc + 2);
  uint64_t items = 1ull << (n - nc - 2);
  LAUNCH(h, k_mcswap, items, (float2*)state, items, P, cmask, t0, t1);
  QS_API_END(h)
}

int qs_apply_mcz(qs_handle_t h, void* state, int n, const int* qubits, int k) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(k >= 1 && k <= QS_MAX_CONTROLS + 1 && k <= n, "mcz needs 1..8 qubits");
  QS_CHECK_ARG(qubits != nullptr, "qubits pointer is null");
  uint64_t mask = 0;
  for (int i = 0; i < k; ++i) { qs_check_qubit(qubits[i], n, "mcz"); mask |= 1ull << qubits[i]; }
  Sorted P = make_sorted(qubits, k);
  uint64_t items = 1ull << (n - k);
  LAUNCH(h, k_mcz, items, (float2*)state, items, P, mask);
  QS_API_END(h)
}

}  // extern "C"
