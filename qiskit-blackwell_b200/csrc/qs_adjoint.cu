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
// of tile-pass launches).  The reverse sweep runs one launch per gate over all
// parameter vectors (grid.y = vector), updates psi and lam in the same pass
// and accumulates the gradient term in FP64 with fixed-order per-vector
// reductions (deterministic).  There is no reference counterpart
// (ROADMAP.md:173-175 lists adjoint differentiation as future work).
#include "qs_api.h"
#include "qs_common.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>

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

  // ---- forward: one circuit per vector, params substituted
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

  // ---- lam = H psi, E = Re<psi|lam>
  // device buffer: grads [nb][nparams] | energies [nb] | partial [nb][256] | U^dag tables
  const size_t ng = (size_t)nb * std::max(nparams, 1);
  const Slice sl = slice(N / 2);
  const Slice sd = slice(N);
  const int nbx = std::max(sl.nbx, sd.nbx);
  size_t bytes = sizeof(double) * (ng + nb + (size_t)nb * nbx) + sizeof(Mat2) * (size_t)nb * nops + 64;
  QS_CUDA(cudaMalloc(&dbuf, bytes));
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
  QS_CUDA(cudaStreamSynchronize(h->stream));
  cudaFree(dbuf);
  dbuf = nullptr;
  qs_batch_plan_destroy(fwd);
  fwd = nullptr;
  return QS_OK;
  }
  catch (const qs_error& e) {
    h->err = e.what();
    cudaStreamSynchronize(h->stream);
    if (dbuf) cudaFree(dbuf);
    if (fwd) qs_batch_plan_destroy(fwd);
    return e.code;
  }
  catch (const std::exception& e) {
    h->err = e.what();
    cudaStreamSynchronize(h->stream);
    if (dbuf) cudaFree(dbuf);
    if (fwd) qs_batch_plan_destroy(fwd);
    return QS_ERR_INVALID;
  }
}
