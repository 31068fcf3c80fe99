// qs_noalloc.cu — an expectation-value entry point that allocates nothing.
//
// qs_expect_pauli_sum stages its Pauli-term table and its per-block partial
// sums in the handle's scratch buffer, which is grown with cudaMalloc on first
// use, and returns the scalar through pinned host memory (cudaMallocHost).
// Some callers cannot have a library allocate device or pinned memory behind
// their back: a runtime that owns every byte of HBM through its own arena and
// budget (a serving process admitting requests against a fixed memory
// budget), or a latency-critical loop that must not pay cudaMalloc/cudaFree's
// implicit device synchronisation.  qs_expect_pauli_sum_noalloc gives them the
// same computation with its scratch in the fixed, file-scope device array
// below; the caller passes the state and receives the value, as before.
//
// Limits and sharing rules:
//   * at most QS_NOALLOC_MAX_TERMS (1024) Pauli terms per call; the block
//     partials never exceed 1024 (the same slicing as qs_expect_pauli_sum);
//   * every GPU that uses it holds the array (about 40 KiB) until the process
//     exits.  With lazy module loading (CUDA_MODULE_LOADING=LAZY, the
//     default) the driver loads this file's module, and so places the array
//     in device memory, at the first call on each device: that first call is
//     the one that takes device memory, so a caller that accounts for every
//     byte makes a warm-up call at start-up;
//   * all calls share it and it keeps the previous call's contents: nothing in
//     it has to start at zero (each call writes the term table, every block's
//     partial and the result before reading them), but calls that overlap on
//     the GPU — two host threads, or two streams — race on it and must be
//     serialised by the caller;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins.  The address is kept for the life of
//     the process: after cudaDeviceReset (which also ends every handle's
//     streams) libqsim must not be used on that device again.
#include "qs_api.h"
#include "qs_common.cuh"
#include <mutex>

namespace {

constexpr int kNAThreads = 256;
constexpr int kNAMaxBlocks = 1024;

struct NATerm { uint64_t x, z; double wr, wi; };

constexpr size_t kTermBytes = sizeof(NATerm) * QS_NOALLOC_MAX_TERMS;  // 32 KiB
constexpr size_t kPartialBytes = sizeof(double) * kNAMaxBlocks;        // 8 KiB
constexpr size_t kScratchBytes = kTermBytes + kPartialBytes + 256;     // + result slot

// The scratch.  In host code this name is only a stand-in for the device
// symbol (handing it to a kernel would fault or address the wrong memory);
// host code uses the device address from cudaGetSymbolAddress instead.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_na_mu;
void* g_na_ptr[64] = {};

// Per-device set-up: the device address of g_noalloc_scratch, looked up once
// with that device current.
void* noalloc_scratch(int device) {
  QS_CHECK_ARG(device >= 0 && device < 64, "device index out of range for the no-alloc scratch");
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_ptr[device]) {
    int cur = -1;
    QS_CUDA(cudaGetDevice(&cur));
    if (cur != device) QS_CUDA(cudaSetDevice(device));
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (cur != device) cudaSetDevice(cur);
    if (e != cudaSuccess)
      throw qs_error(QS_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
    g_na_ptr[device] = p;
  }
  return g_na_ptr[device];
}

__device__ __forceinline__ double na_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double na_block_sum(double v) {
  __shared__ double ws[32];
  v = na_warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = 0.0;
  if (w == 0) {
    v = lane < nw ? ws[lane] : 0.0;
    v = na_warp_sum(v);
  }
  return v;
}

// Stage 1: per-block partials of sum_i Re(conj(psi_i) (H psi)_i), terms and
// partials addressed inside the static scratch.
__global__ void k_pauli_expect_na(const float2* __restrict__ s, uint64_t n, const NATerm* __restrict__ terms,
                                  int nterms, uint64_t per, double* __restrict__ partial) {
  extern __shared__ NATerm st[];
  for (int k = threadIdx.x; k < nterms; k += blockDim.x) st[k] = terms[k];
  __syncthreads();
  const uint64_t b0 = (uint64_t)blockIdx.x * per;
  const uint64_t e = min(b0 + per, n);
  double acc = 0.0;
  for (uint64_t i = b0 + threadIdx.x; i < e; i += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nterms; ++k) {
      const NATerm T = st[k];
      const uint64_t j = i ^ T.x;
      const float2 b = s[j];
      const double sg = (__popcll(j & T.z) & 1) ? -1.0 : 1.0;
      re += sg * (T.wr * b.x - T.wi * b.y);
      im += sg * (T.wr * b.y + T.wi * b.x);
    }
    const float2 a = s[i];
    acc += (double)a.x * re + (double)a.y * im;
  }
  acc = na_block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// Stage 2: one block sums the partials in a fixed order into *result.
__global__ void k_final_na(const double* __restrict__ partial, int nb, double* __restrict__ result) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += partial[i];
  acc = na_block_sum(acc);
  if (threadIdx.x == 0) *result = acc;
}

}  // namespace

extern "C" int qs_expect_pauli_sum_noalloc(qs_handle_t h, const void* state, int n, const uint64_t* x,
                                           const uint64_t* z, const double* c, int nterms, double* out_host) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(out_host != nullptr, "out is null");
  QS_CHECK_ARG(x && z && c, "term pointers are null");
  if (nterms < 1 || nterms > QS_NOALLOC_MAX_TERMS)
    throw qs_error(QS_ERR_INVALID, "n_terms must be in [1, " + std::to_string(QS_NOALLOC_MAX_TERMS) +
                                       "] for the no-alloc expectation (its scratch is a fixed static array)");
  char* base = static_cast<char*>(noalloc_scratch(h->device));
  NATerm* d_terms = reinterpret_cast<NATerm*>(base);
  double* d_partial = reinterpret_cast<double*>(base + kTermBytes);
  double* d_result = reinterpret_cast<double*>(base + kTermBytes + kPartialBytes);

  // Term table on the host stack (no heap, no pinned memory), then into the
  // static scratch.  A pageable source is staged by the driver before the
  // call returns, so the stack array may go out of scope afterwards.
  NATerm T[QS_NOALLOC_MAX_TERMS];
  const uint64_t lim = (1ull << n) - 1ull;
  static const double pr[4] = {1, 0, -1, 0}, pim[4] = {0, 1, 0, -1};
  for (int k = 0; k < nterms; ++k) {
    QS_CHECK_ARG((x[k] & ~lim) == 0 && (z[k] & ~lim) == 0, "Pauli mask has bits beyond n_qubits");
    const int ny = __builtin_popcountll(x[k] & z[k]) & 3;
    T[k] = NATerm{x[k], z[k], c[k] * pr[ny], c[k] * pim[ny]};
  }
  QS_CUDA(cudaMemcpyAsync(d_terms, T, sizeof(NATerm) * nterms, cudaMemcpyHostToDevice, h->stream));

  // Same slicing as qs_expect_pauli_sum (at most 1024 blocks).
  const uint64_t N = 1ull << n;
  uint64_t nb = (N + 4095) / 4096;
  if (nb > kNAMaxBlocks) nb = kNAMaxBlocks;
  if (nb < 1) nb = 1;
  const uint64_t per = (N + nb - 1) / nb;
  k_pauli_expect_na<<<(unsigned)nb, kNAThreads, sizeof(NATerm) * nterms, h->stream>>>(
      (const float2*)state, N, d_terms, nterms, per, d_partial);
  qs_after_launch(h, "k_pauli_expect_na");
  k_final_na<<<1, 1024, 0, h->stream>>>(d_partial, (int)nb, d_result);
  qs_after_launch(h, "k_final_na");
  QS_CUDA(cudaMemcpyAsync(out_host, d_result, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaStreamSynchronize(h->stream));
  QS_API_END(h)
}
