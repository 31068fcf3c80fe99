// qs_common.cuh — device helpers shared by the libqsim kernels.
//
// Complex64 amplitudes are float2 (x = re, y = im).  All index arithmetic is
// 64-bit so that 2^32-amplitude states (32 qubits, 32 GiB) are addressable.
//
// Compensated arithmetic uses the __fmul_rn/__fadd_rn/__fsub_rn intrinsics,
// which nvcc never contracts into FMAs, together with explicit fmaf, so that
// the error-free transformations below stay exact under the default
// -fmad=true.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qs {

// Programmatic dependent launch (kernels launched with qs_launch_pdl): wait
// for the grid before this one in the stream (griddepcontrol.wait: it has
// finished and its writes are visible; a no-op for a kernel launched without
// the attribute), then let the next grid begin its launch, whose CTAs wait in
// turn before they touch memory.  Called first thing by such a kernel.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ------------------------------------------------------------ indices -----
// Insert a zero bit at position q: bits >= q move up by one.
__device__ __forceinline__ uint64_t insert_zero(uint64_t x, int q) {
  uint64_t lo = x & ((1ull << q) - 1ull);
  return ((x ^ lo) << 1) | lo;
}

// Insert zeros at k ascending positions.
__device__ __forceinline__ uint64_t insert_zeros(uint64_t x, const int* q, int k) {
  for (int j = 0; j < k; ++j) x = insert_zero(x, q[j]);
  return x;
}

// -------------------------------------------------- error-free products ---
// TwoProduct (Dekker; with FMA as in Ogita, Rump, Oishi, "Accurate Sum and
// Dot Product", SIAM J. Sci. Comput. 26(6), 2005, Algorithm 3.5):
// a*b = p + e exactly.
__device__ __forceinline__ void two_prod(float a, float b, float& p, float& e) {
  p = __fmul_rn(a, b);
  e = fmaf(a, b, -p);
}

// TwoSum (Knuth, TAOCP vol. 2, 4.2.2): a+b = s + e exactly.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  float z = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, z)), __fsub_rn(b, z));
}

// Dot2 (Ogita-Rump-Oishi 2005, Algorithm 5.3): sum_k x_k*y_k evaluated as if
// in twice the working precision, then rounded once.
template <int K>
__device__ __forceinline__ float dot2(const float (&x)[K], const float (&y)[K]) {
  float s, c;
  two_prod(x[0], y[0], s, c);
#pragma unroll
  for (int k = 1; k < K; ++k) {
    float p, e, q;
    two_prod(x[k], y[k], p, e);
    two_sum(s, p, s, q);
    c = __fadd_rn(c, __fadd_rn(q, e));
  }
  return __fadd_rn(s, c);
}

// Compensated complex product a*b.  Each component is a 2x2 determinant-like
// expression evaluated with Kahan's FMA method (W. Kahan; error analysis in
// Jeannerod, Louvet, Muller, "Further analysis of Kahan's algorithm for the
// accurate computation of 2x2 determinants", Math. Comp. 82, 2013): at most
// ~1.5 ulp, and exact when b is 0, +-1 or +-i.
__device__ __forceinline__ float kahan_ab_minus_cd(float a, float b, float c, float d) {
  float w = __fmul_rn(c, d);
  float e = fmaf(-c, d, w);
  float f = fmaf(a, b, -w);
  return __fadd_rn(f, e);
}
__device__ __forceinline__ float2 cmul_comp(float2 a, float2 b) {
  return make_float2(kahan_ab_minus_cd(a.x, b.x, a.y, b.y),
                     kahan_ab_minus_cd(a.x, b.y, -a.y, b.x));
}

// Compensated sum_k g_k * a_k over K complex terms (Dot2 per component).
template <int K>
__device__ __forceinline__ float2 cdot_comp(const float2 (&g)[K], const float2 (&a)[K]) {
  float xr[2 * K], yr[2 * K], xi[2 * K], yi[2 * K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    xr[2 * k] = g[k].x;  yr[2 * k] = a[k].x;
    xr[2 * k + 1] = -g[k].y; yr[2 * k + 1] = a[k].y;
    xi[2 * k] = g[k].x;  yi[2 * k] = a[k].y;
    xi[2 * k + 1] = g[k].y; yi[2 * k + 1] = a[k].x;
  }
  return make_float2(dot2<2 * K>(xr, yr), dot2<2 * K>(xi, yi));
}

// ----------------------------------------------------- fast FMA chains ----
// g0*a0 + g1*a1 as an FMA chain (used inside the fused tile pass, where the
// work is FP32-pipe bound; each FMA rounds once).
__device__ __forceinline__ float2 cfma2(float2 g0, float2 a0, float2 g1, float2 a1) {
  float re = __fmul_rn(g0.x, a0.x);
  re = fmaf(-g0.y, a0.y, re);
  re = fmaf(g1.x, a1.x, re);
  re = fmaf(-g1.y, a1.y, re);
  float im = __fmul_rn(g0.x, a0.y);
  im = fmaf(g0.y, a0.x, im);
  im = fmaf(g1.x, a1.y, im);
  im = fmaf(g1.y, a1.x, im);
  return make_float2(re, im);
}

__device__ __forceinline__ float2 cfma4(const float2* g, float2 a0, float2 a1, float2 a2, float2 a3) {
  float re = __fmul_rn(g[0].x, a0.x);
  re = fmaf(-g[0].y, a0.y, re);
  re = fmaf(g[1].x, a1.x, re);
  re = fmaf(-g[1].y, a1.y, re);
  re = fmaf(g[2].x, a2.x, re);
  re = fmaf(-g[2].y, a2.y, re);
  re = fmaf(g[3].x, a3.x, re);
  re = fmaf(-g[3].y, a3.y, re);
  float im = __fmul_rn(g[0].x, a0.y);
  im = fmaf(g[0].y, a0.x, im);
  im = fmaf(g[1].x, a1.y, im);
  im = fmaf(g[1].y, a1.x, im);
  im = fmaf(g[2].x, a2.y, im);
  im = fmaf(g[2].y, a2.x, im);
  im = fmaf(g[3].x, a3.y, im);
  im = fmaf(g[3].y, a3.x, im);
  return make_float2(re, im);
}

// ------------------------------------------------------ vector memory -----
__device__ __forceinline__ float4 ld4(const float2* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float2* p, float2 a, float2 b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// Grid-stride loop bounds.
__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

}  // namespace qs
