// qs_cheb.cu — CSR SpMV and the Chebyshev recurrence for exp(-iHt)|psi>.
//
// Rows are processed by V-lane sub-warps (V = 4..32, picked from the mean row
// length) so that the col_idx/values streams are read coalesced.  Each lane
// accumulates its entries with error-free products and TwoSum (a compensated
// "Kahan" row sum); lanes are combined in a fixed shuffle order, also
// compensated, so results are deterministic.
//
// The fused recurrence kernel does, per degree k and row r, in one launch:
//     t      = 2 * scale * (A x_{k})_r - x_{k-1,r}      (x_{k+1}, in place of x_{k-1})
//     out_r += c_{k+1} * t
// which needs three vectors instead of the reference's five
// (blackwell_backend/chebyshev.py:117-123).
#include "qs_api.h"
#include "qs_common.cuh"
#include <algorithm>
#include <vector>

using namespace qs;

namespace {

constexpr int kThreads = 256;

struct Acc { float s, c; };  // compensated sum: value = s + c

__device__ __forceinline__ void acc_add_prod(Acc& a, float x, float y) {
  float p, e, q;
  two_prod(x, y, p, e);
  two_sum(a.s, p, a.s, q);
  a.c = __fadd_rn(a.c, __fadd_rn(q, e));
}

template <int V>
__device__ __forceinline__ Acc acc_reduce(Acc a) {
#pragma unroll
  for (int o = V / 2; o > 0; o >>= 1) {
    float s2 = __shfl_down_sync(0xffffffffu, a.s, o, V);
    float c2 = __shfl_down_sync(0xffffffffu, a.c, o, V);
    float s, e;
    two_sum(a.s, s2, s, e);
    a.s = s;
    a.c = __fadd_rn(__fadd_rn(a.c, c2), e);
  }
  return a;
}

// Compensated row dot: returns (A x)_r for the row handled by this sub-warp.
// r < 0 means "no row": the lanes still take part in the shuffles.
template <int V>
__device__ __forceinline__ float2 row_dot(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                          const float2* __restrict__ val, const float2* __restrict__ x, int64_t r,
                                          int lane) {
  int32_t b = 0, e = 0;
  if (r >= 0) { b = rp[r]; e = rp[r + 1]; }
  Acc re{0.f, 0.f}, im{0.f, 0.f};
  for (int32_t j = b + lane; j < e; j += V) {
    const float2 v = val[j];
    const float2 xj = x[ci[j]];
    acc_add_prod(re, v.x, xj.x);
    acc_add_prod(re, -v.y, xj.y);
    acc_add_prod(im, v.x, xj.y);
    acc_add_prod(im, v.y, xj.x);
  }
  re = acc_reduce<V>(re);
  im = acc_reduce<V>(im);
  return make_float2(__fadd_rn(re.s, re.c), __fadd_rn(im.s, im.c));
}

// Warp-uniform row loop: every warp handles 32/V consecutive rows per
// iteration, so all 32 lanes always execute the same shuffles.
#define ROW_LOOP(V, ...)                                                        \
  const int lane = threadIdx.x & (V - 1);                                        \
  const int sub = (threadIdx.x & 31) / V;                                        \
  const int64_t warp = (int64_t)(gtid() >> 5), nwarps = (int64_t)(gstride() >> 5); \
  constexpr int rpw = 32 / V;                                                    \
  for (int64_t base = warp * rpw; base < nrows; base += nwarps * rpw) {          \
    const int64_t r = base + sub;                                                \
    const bool live = r < nrows;                                                 \
    __VA_ARGS__                                                                  \
  }

template <int V>
__global__ void k_spmv(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const float2* __restrict__ val,
                       int64_t nrows, const float2* __restrict__ x, float2* __restrict__ y, float2 alpha,
                       float2 beta) {
  pdl_begin();
  ROW_LOOP(V, {
    const float2 d = row_dot<V>(rp, ci, val, x, live ? r : -1, lane);
    if (live && lane == 0) {
      const float2 yo = y[r];
      float2 o;
      o.x = alpha.x * d.x - alpha.y * d.y + (beta.x * yo.x - beta.y * yo.y);
      o.y = alpha.x * d.y + alpha.y * d.x + (beta.x * yo.y + beta.y * yo.x);
      y[r] = o;
    }
  })
}

// Fused Chebyshev degree step.  xprev is overwritten with x_next.
template <int V>
__global__ void k_cheb_fused(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             const float2* __restrict__ val, int64_t nrows, const float2* __restrict__ xk,
                             float2* __restrict__ xprev, float2* __restrict__ out, float two_scale, float2 c) {
  pdl_begin();
  ROW_LOOP(V, {
    const float2 d = row_dot<V>(rp, ci, val, xk, live ? r : -1, lane);
    if (live && lane == 0) {
      const float2 p = xprev[r];
      const float2 t = make_float2(fmaf(two_scale, d.x, -p.x), fmaf(two_scale, d.y, -p.y));
      xprev[r] = t;
      float2 a = out[r];
      a.x = fmaf(c.x, t.x, fmaf(-c.y, t.y, a.x));
      a.y = fmaf(c.x, t.y, fmaf(c.y, t.x, a.y));
      out[r] = a;
    }
  })
}

// x1 = scale * A x0 ; out = c0 * x0 + c1 * x1
template <int V>
__global__ void k_cheb_first(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             const float2* __restrict__ val, int64_t nrows, const float2* __restrict__ x0,
                             float2* __restrict__ x1, float2* __restrict__ out, float scale, float2 c0, float2 c1) {
  pdl_begin();
  ROW_LOOP(V, {
    const float2 d = row_dot<V>(rp, ci, val, x0, live ? r : -1, lane);
    if (live && lane == 0) {
      const float2 t = make_float2(scale * d.x, scale * d.y);
      x1[r] = t;
      const float2 a0 = x0[r];
      float2 a;
      a.x = c0.x * a0.x - c0.y * a0.y;
      a.y = c0.x * a0.y + c0.y * a0.x;
      a.x = fmaf(c1.x, t.x, fmaf(-c1.y, t.y, a.x));
      a.y = fmaf(c1.x, t.y, fmaf(c1.y, t.x, a.y));
      out[r] = a;
    }
  })
}

// ---- reference mirrors (chebyshev_sm120.cu:24-91): float4 elementwise ----
__global__ void k_step(const float4* __restrict__ s, const float4* __restrict__ p, float4* __restrict__ nx, uint64_t nv) {
  pdl_begin();
  for (uint64_t i = gtid(); i < nv; i += gstride()) {
    float4 a = s[i], b = p[i];
    nx[i] = make_float4(2.f * a.x - b.x, 2.f * a.y - b.y, 2.f * a.z - b.z, 2.f * a.w - b.w);
  }
}
__global__ void k_accum(float4* __restrict__ acc, const float4* __restrict__ t, float2 c, uint64_t nv) {
  pdl_begin();
  for (uint64_t i = gtid(); i < nv; i += gstride()) {
    float4 a = acc[i], x = t[i];
    a.x += c.x * x.x - c.y * x.y;
    a.y += c.x * x.y + c.y * x.x;
    a.z += c.x * x.z - c.y * x.w;
    a.w += c.x * x.w + c.y * x.z;
    acc[i] = a;
  }
}
__global__ void k_step_accum(const float4* __restrict__ s, const float4* __restrict__ p, float4* __restrict__ nx,
                             float4* __restrict__ acc, float2 c, uint64_t nv) {
  pdl_begin();
  for (uint64_t i = gtid(); i < nv; i += gstride()) {
    float4 a = s[i], b = p[i], r = acc[i];
    float4 t = make_float4(2.f * a.x - b.x, 2.f * a.y - b.y, 2.f * a.z - b.z, 2.f * a.w - b.w);
    r.x += c.x * t.x - c.y * t.y;
    r.y += c.x * t.y + c.y * t.x;
    r.z += c.x * t.z - c.y * t.w;
    r.w += c.x * t.w + c.y * t.z;
    nx[i] = t;
    acc[i] = r;
  }
}

// ---- matrix-free Pauli-sum operator -------------------------------------
// (H x)_i = sum_t w_t (-1)^{popc((i^x_t) & z_t)} x[i ^ x_t],  w_t = c_t i^{|x_t&z_t|}.
// Terms live in shared memory; XOR with a constant maps aligned blocks onto
// aligned blocks, so the gathers of a warp stay coalesced.
struct __align__(16) PTerm { uint64_t x, z; float wr, wi, pad0, pad1; };

__device__ __forceinline__ float2 hx_row(const PTerm* __restrict__ st, int nterms, const float2* __restrict__ x,
                                         uint64_t i) {
  float re = 0.f, im = 0.f;
  for (int k = 0; k < nterms; ++k) {
    const PTerm T = st[k];
    const uint64_t j = i ^ T.x;
    const float2 v = x[j];
    const float sg = (__popcll(j & T.z) & 1) ? -1.f : 1.f;
    const float wr = sg * T.wr, wi = sg * T.wi;
    re = fmaf(wr, v.x, fmaf(-wi, v.y, re));
    im = fmaf(wr, v.y, fmaf(wi, v.x, im));
  }
  return make_float2(re, im);
}

__global__ void k_chebp_first(const PTerm* __restrict__ terms, int nterms, uint64_t n, const float2* __restrict__ x0,
                              float2* __restrict__ x1, float2* __restrict__ out, float scale, float2 c0, float2 c1) {
  pdl_begin();
  extern __shared__ PTerm st[];
  for (int k = threadIdx.x; k < nterms; k += blockDim.x) st[k] = terms[k];
  __syncthreads();
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const float2 d = hx_row(st, nterms, x0, i);
    const float2 t = make_float2(scale * d.x, scale * d.y);
    x1[i] = t;
    const float2 a0 = x0[i];
    float2 a;
    a.x = c0.x * a0.x - c0.y * a0.y;
    a.y = c0.x * a0.y + c0.y * a0.x;
    a.x = fmaf(c1.x, t.x, fmaf(-c1.y, t.y, a.x));
    a.y = fmaf(c1.x, t.y, fmaf(c1.y, t.x, a.y));
    out[i] = a;
  }
}

__global__ void k_chebp_fused(const PTerm* __restrict__ terms, int nterms, uint64_t n, const float2* __restrict__ xk,
                              float2* __restrict__ xprev, float2* __restrict__ out, float two_scale, float2 c) {
  pdl_begin();
  extern __shared__ PTerm st[];
  for (int k = threadIdx.x; k < nterms; k += blockDim.x) st[k] = terms[k];
  __syncthreads();
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const float2 d = hx_row(st, nterms, xk, i);
    const float2 p = xprev[i];
    const float2 t = make_float2(fmaf(two_scale, d.x, -p.x), fmaf(two_scale, d.y, -p.y));
    xprev[i] = t;
    float2 a = out[i];
    a.x = fmaf(c.x, t.x, fmaf(-c.y, t.y, a.x));
    a.y = fmaf(c.x, t.y, fmaf(c.y, t.x, a.y));
    out[i] = a;
  }
}

// Up to 32 qubits the matrix-free recurrence uses 32-bit indices and splits
// H into its diagonal and off-diagonal parts:
//   * terms with x_t = 0 sum to a real diagonal D_i = sum_t c_t (-1)^{popc(i & z_t)},
//     tabulated once per evolution (FP64 sums rounded to FP32, 4 B per
//     amplitude), so the degree loop reads D_i instead of evaluating them;
//   * the other terms are sorted by X mask and paired: both terms of a pair
//     share one gather x[i ^ x] (e.g. X_a X_b and Y_a Y_b), and a lone term
//     has a zero partner.  The sign (-1)^{popc(j & z)} is applied by flipping
//     the sign bit of the weight.
struct __align__(16) PPair { uint32_t x, z0, z1, pad; float w0r, w0i, w1r, w1i; };
struct __align__(16) PDiag { uint64_t z; double c; };

__global__ void k_chebp_diag(const PDiag* __restrict__ terms, int nterms, uint64_t n, float* __restrict__ D) {
  pdl_begin();
  extern __shared__ PDiag sd[];
  for (int k = threadIdx.x; k < nterms; k += blockDim.x) sd[k] = terms[k];
  __syncthreads();
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    double d = 0.0;
    for (int k = 0; k < nterms; ++k) d += (__popcll(i & sd[k].z) & 1) ? -sd[k].c : sd[k].c;
    D[i] = (float)d;
  }
}

__device__ __forceinline__ float flip_if(float w, uint32_t sbit) { return __int_as_float(__float_as_int(w) ^ sbit); }

__device__ __forceinline__ float2 hx_row_pairs(const PPair* __restrict__ st, int npairs, const float2* __restrict__ x,
                                               const float* __restrict__ D, uint32_t i) {
  float re = 0.f, im = 0.f;
  if (D) {
    const float d = D[i];
    const float2 v = x[i];
    re = d * v.x;
    im = d * v.y;
  }
  for (int k = 0; k < npairs; ++k) {
    const PPair P = st[k];
    const uint32_t j = i ^ P.x;
    const float2 v = x[j];
    const uint32_t s0 = (uint32_t)(__popc(j & P.z0) & 1) << 31, s1 = (uint32_t)(__popc(j & P.z1) & 1) << 31;
    const float wr = flip_if(P.w0r, s0) + flip_if(P.w1r, s1);
    const float wi = flip_if(P.w0i, s0) + flip_if(P.w1i, s1);
    re = fmaf(wr, v.x, fmaf(-wi, v.y, re));
    im = fmaf(wr, v.y, fmaf(wi, v.x, im));
  }
  return make_float2(re, im);
}

__global__ void k_chebp_first_pairs(const PPair* __restrict__ pairs, int npairs, uint64_t n,
                                    const float* __restrict__ D, const float2* __restrict__ x0,
                                    float2* __restrict__ x1, float2* __restrict__ out, float scale, float2 c0,
                                    float2 c1) {
  pdl_begin();
  extern __shared__ PPair sp[];
  for (int k = threadIdx.x; k < npairs; k += blockDim.x) sp[k] = pairs[k];
  __syncthreads();
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const float2 d = hx_row_pairs(sp, npairs, x0, D, (uint32_t)i);
    const float2 t = make_float2(scale * d.x, scale * d.y);
    x1[i] = t;
    const float2 a0 = x0[i];
    float2 a;
    a.x = c0.x * a0.x - c0.y * a0.y;
    a.y = c0.x * a0.y + c0.y * a0.x;
    a.x = fmaf(c1.x, t.x, fmaf(-c1.y, t.y, a.x));
    a.y = fmaf(c1.x, t.y, fmaf(c1.y, t.x, a.y));
    out[i] = a;
  }
}

__global__ void k_chebp_fused_pairs(const PPair* __restrict__ pairs, int npairs, uint64_t n,
                                    const float* __restrict__ D, const float2* __restrict__ xk,
                                    float2* __restrict__ xprev, float2* __restrict__ out, float two_scale,
                                    float2 c) {
  pdl_begin();
  extern __shared__ PPair sp[];
  for (int k = threadIdx.x; k < npairs; k += blockDim.x) sp[k] = pairs[k];
  __syncthreads();
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const float2 d = hx_row_pairs(sp, npairs, xk, D, (uint32_t)i);
    const float2 p = xprev[i];
    const float2 t = make_float2(fmaf(two_scale, d.x, -p.x), fmaf(two_scale, d.y, -p.y));
    xprev[i] = t;
    float2 a = out[i];
    a.x = fmaf(c.x, t.x, fmaf(-c.y, t.y, a.x));
    a.y = fmaf(c.x, t.y, fmaf(c.y, t.x, a.y));
    out[i] = a;
  }
}

int pick_V(int64_t nrows, const int32_t* rp_dev, qs_context* h) {
  // mean row length from the first and last row pointers
  int32_t ends[2] = {0, 0};
  QS_CUDA(cudaMemcpyAsync(&ends[0], rp_dev, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaMemcpyAsync(&ends[1], rp_dev + nrows, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaStreamSynchronize(h->stream));
  const double mean = nrows > 0 ? double(ends[1] - ends[0]) / double(nrows) : 1.0;
  if (mean <= 6) return 4;
  if (mean <= 12) return 8;
  if (mean <= 28) return 16;
  return 32;
}

#define DISPATCH_V(V, KERN, GRID, ...)                                            \
  switch (V) {                                                                   \
    case 4: qs_launch_pdl(h, KERN<4>, dim3(GRID), dim3(kThreads), 0, __VA_ARGS__); break;       \
    case 8: qs_launch_pdl(h, KERN<8>, dim3(GRID), dim3(kThreads), 0, __VA_ARGS__); break;       \
    case 16: qs_launch_pdl(h, KERN<16>, dim3(GRID), dim3(kThreads), 0, __VA_ARGS__); break;     \
    default: qs_launch_pdl(h, KERN<32>, dim3(GRID), dim3(kThreads), 0, __VA_ARGS__); break;     \
  }

inline void check_vec(const void* p, const char* what) {
  if (!p || ((uintptr_t)p & 15u)) throw qs_error(QS_ERR_INVALID, std::string(what) + " must be a 16-byte aligned device pointer");
}

}  // namespace

extern "C" {

int qs_spmv_csr(qs_handle_t h, const int32_t* rp, const int32_t* ci, const void* val, int64_t nrows, const void* x,
                void* y, double ar, double ai, double br, double bi) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(rp && ci && val && x && y, "null CSR or vector pointer");
  QS_CHECK_ARG(nrows >= 0, "n_rows must be >= 0");
  QS_CHECK_ARG(x != y, "x and y must not alias");
  if (nrows == 0) return QS_OK;
  const int V = pick_V(nrows, rp, h);
  const unsigned grid = (unsigned)qs_blocks_for(h, (uint64_t)nrows * V, kThreads, 16);
  DISPATCH_V(V, k_spmv, grid, rp, ci, (const float2*)val, nrows, (const float2*)x, (float2*)y,
             make_float2((float)ar, (float)ai), make_float2((float)br, (float)bi));
  qs_after_launch(h, "k_spmv");
  QS_API_END(h)
}

int qs_cheb_step(qs_handle_t h, const void* s, const void* p, void* nx, int64_t n) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  check_vec(s, "spmv_result"); check_vec(p, "t_prev"); check_vec(nx, "t_next");
  QS_CHECK_ARG(n >= 0 && (n & 1) == 0, "n must be even and >= 0");
  const uint64_t nv = (uint64_t)n / 2;
  if (nv) {
    qs_launch_pdl(h, k_step, dim3(qs_blocks_for(h, nv, kThreads)), dim3(kThreads), 0, (const float4*)s, (const float4*)p, (float4*)nx, nv);
    qs_after_launch(h, "k_step");
  }
  QS_API_END(h)
}

int qs_cheb_accum(qs_handle_t h, void* acc, const void* t, double cr, double ci_, int64_t n) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  check_vec(acc, "accum"); check_vec(t, "t_k");
  QS_CHECK_ARG(n >= 0 && (n & 1) == 0, "n must be even and >= 0");
  const uint64_t nv = (uint64_t)n / 2;
  if (nv) {
    qs_launch_pdl(h, k_accum, dim3(qs_blocks_for(h, nv, kThreads)), dim3(kThreads), 0, (float4*)acc, (const float4*)t,
                                                                        make_float2((float)cr, (float)ci_), nv);
    qs_after_launch(h, "k_accum");
  }
  QS_API_END(h)
}

int qs_cheb_step_accum(qs_handle_t h, const void* s, const void* p, void* nx, void* acc, double cr, double ci_,
                       int64_t n) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  check_vec(s, "spmv_result"); check_vec(p, "t_prev"); check_vec(nx, "t_next"); check_vec(acc, "accum");
  QS_CHECK_ARG(n >= 0 && (n & 1) == 0, "n must be even and >= 0");
  const uint64_t nv = (uint64_t)n / 2;
  if (nv) {
    qs_launch_pdl(h, k_step_accum, dim3(qs_blocks_for(h, nv, kThreads)), dim3(kThreads), 0, 
        (const float4*)s, (const float4*)p, (float4*)nx, (float4*)acc, make_float2((float)cr, (float)ci_), nv);
    qs_after_launch(h, "k_step_accum");
  }
  QS_API_END(h)
}

int qs_cheb_evolve(qs_handle_t h, const int32_t* rp, const int32_t* ci, const void* val, int n, const void* psi,
                   void* out, const double* coeffs, int K, double scale, void* work) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(psi, n);
  qs_check_state(out, n);
  qs_check_state(work, n);
  QS_CHECK_ARG(rp && ci && val && coeffs, "null CSR or coefficient pointer");
  QS_CHECK_ARG(K >= 1, "K must be >= 1");
  const int64_t N = (int64_t)1 << n;
  float2* x0 = (float2*)work;        // x_{k-1}
  float2* x1 = x0 + N;               // x_k
  QS_CUDA(cudaMemcpyAsync(x0, psi, sizeof(float2) * N, cudaMemcpyDeviceToDevice, h->stream));
  const int V = pick_V(N, rp, h);
  const unsigned grid = (unsigned)qs_blocks_for(h, (uint64_t)N * V, kThreads, 16);
  auto C = [&](int k) { return make_float2((float)coeffs[2 * k], (float)coeffs[2 * k + 1]); };
  DISPATCH_V(V, k_cheb_first, grid, rp, ci, (const float2*)val, N, x0, x1, (float2*)out, (float)scale, C(0), C(1));
  qs_after_launch(h, "k_cheb_first");
  const float two_scale = (float)(2.0 * scale);
  for (int k = 2; k <= K; ++k) {
    // x0 holds x_{k-2}, x1 holds x_{k-1}; x0 becomes x_k
    DISPATCH_V(V, k_cheb_fused, grid, rp, ci, (const float2*)val, N, x1, x0, (float2*)out, two_scale, C(k));
    qs_after_launch(h, "k_cheb_fused");
    std::swap(x0, x1);
  }
  QS_API_END(h)
}

int qs_cheb_evolve_pauli(qs_handle_t h, int n, const void* psi, void* out, const uint64_t* xm, const uint64_t* zm,
                         const double* coefs, int nterms, const double* coeffs, int K, double scale, void* work) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(psi, n);
  qs_check_state(out, n);
  qs_check_state(work, n);
  QS_CHECK_ARG(xm && zm && coefs && coeffs, "null term or coefficient pointer");
  QS_CHECK_ARG(nterms >= 1 && nterms <= 1024, "n_terms must be in [1, 1024]");
  QS_CHECK_ARG(K >= 1, "K must be >= 1");
  const uint64_t lim = (1ull << n) - 1ull;
  std::vector<PTerm> T(nterms);
  static const float pr[4] = {1.f, 0.f, -1.f, 0.f}, pim[4] = {0.f, 1.f, 0.f, -1.f};
  for (int k = 0; k < nterms; ++k) {
    QS_CHECK_ARG((xm[k] & ~lim) == 0 && (zm[k] & ~lim) == 0, "Pauli mask has bits beyond n_qubits");
    const int ny = __builtin_popcountll(xm[k] & zm[k]) & 3;
    T[k] = PTerm{xm[k], zm[k], (float)(coefs[k] * pr[ny]), (float)(coefs[k] * pim[ny]), 0.f, 0.f};
  }
  const uint64_t N = 1ull << n;
  float2* x0 = (float2*)work;
  float2* x1 = x0 + N;
  auto C = [&](int k) { return make_float2((float)coeffs[2 * k], (float)coeffs[2 * k + 1]); };
  const float two_scale = (float)(2.0 * scale);
  if (n <= 32) {
    // diagonal terms and X-mask pairs (see PPair)
    std::vector<PDiag> dg;
    std::vector<int> off;
    for (int k = 0; k < nterms; ++k) {
      if (xm[k] == 0) dg.push_back(PDiag{zm[k], coefs[k]});
      else off.push_back(k);
    }
    std::stable_sort(off.begin(), off.end(), [&](int a, int b) { return xm[a] < xm[b]; });
    std::vector<PPair> pr;
    for (size_t u = 0; u < off.size();) {
      const PTerm& A = T[off[u]];
      PPair P{(uint32_t)A.x, (uint32_t)A.z, 0u, 0u, A.wr, A.wi, 0.f, 0.f};
      if (u + 1 < off.size() && xm[off[u + 1]] == xm[off[u]]) {
        const PTerm& B = T[off[u + 1]];
        P.z1 = (uint32_t)B.z;
        P.w1r = B.wr;
        P.w1i = B.wi;
        u += 2;
      } else {
        u += 1;
      }
      pr.push_back(P);
    }
    const size_t pbytes = sizeof(PPair) * pr.size(), dbytes = sizeof(PDiag) * dg.size();
    char* dmem = (char*)h->scratch_get(std::max<size_t>(16, pbytes + dbytes));
    const PPair* dP = (const PPair*)dmem;
    const PDiag* dD = (const PDiag*)(dmem + pbytes);
    if (pbytes) QS_CUDA(cudaMemcpyAsync(dmem, pr.data(), pbytes, cudaMemcpyHostToDevice, h->stream));
    if (dbytes) QS_CUDA(cudaMemcpyAsync(dmem + pbytes, dg.data(), dbytes, cudaMemcpyHostToDevice, h->stream));
    float* D = nullptr;
    if (!dg.empty()) {
      QS_CUDA(cudaMallocAsync((void**)&D, sizeof(float) * N, h->stream));
      qs_launch_pdl(h, k_chebp_diag, dim3(qs_blocks_for(h, N, kThreads)), dim3(kThreads), dbytes, dD, (int)dg.size(), N, D);
      qs_after_launch(h, "k_chebp_diag");
    }
    try {
      QS_CUDA(cudaMemcpyAsync(x0, psi, sizeof(float2) * N, cudaMemcpyDeviceToDevice, h->stream));
      const unsigned grid = (unsigned)qs_blocks_for(h, N, kThreads, 8);
      const int np = (int)pr.size();
      qs_launch_pdl(h, k_chebp_first_pairs, dim3(grid), dim3(kThreads), pbytes, dP, np, N, D, x0, x1, (float2*)out,
                                                                 (float)scale, C(0), C(1));
      qs_after_launch(h, "k_chebp_first_pairs");
      for (int k = 2; k <= K; ++k) {
        qs_launch_pdl(h, k_chebp_fused_pairs, dim3(grid), dim3(kThreads), pbytes, dP, np, N, D, x1, x0, (float2*)out,
                                                                   two_scale, C(k));
        qs_after_launch(h, "k_chebp_fused_pairs");
        std::swap(x0, x1);
      }
    } catch (...) {
      if (D) cudaFreeAsync(D, h->stream);
      throw;
    }
    if (D) QS_CUDA(cudaFreeAsync(D, h->stream));
    return QS_OK;
  }
  PTerm* dT = (PTerm*)h->scratch_get(sizeof(PTerm) * nterms);
  QS_CUDA(cudaMemcpyAsync(dT, T.data(), sizeof(PTerm) * nterms, cudaMemcpyHostToDevice, h->stream));
  QS_CUDA(cudaMemcpyAsync(x0, psi, sizeof(float2) * N, cudaMemcpyDeviceToDevice, h->stream));
  const unsigned grid = (unsigned)qs_blocks_for(h, N, kThreads, 8);
  const size_t smem = sizeof(PTerm) * nterms;
  qs_launch_pdl(h, k_chebp_first, dim3(grid), dim3(kThreads), smem, dT, nterms, N, x0, x1, (float2*)out, (float)scale, C(0), C(1));
  qs_after_launch(h, "k_chebp_first");
  for (int k = 2; k <= K; ++k) {
    qs_launch_pdl(h, k_chebp_fused, dim3(grid), dim3(kThreads), smem, dT, nterms, N, x1, x0, (float2*)out, two_scale, C(k));
    qs_after_launch(h, "k_chebp_fused");
    std::swap(x0, x1);
  }
  QS_API_END(h)
}

}  // extern "C"
