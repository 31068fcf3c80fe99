// qs_context.cu — handle lifecycle, streams, scratch and error reporting.
#include "qs_api.h"
#include <atomic>
#include <cstring>
#include <cstdlib>
#include <set>
#include <mutex>

static thread_local std::string g_tls_err;
void qs_set_tls_error(const std::string& m) { g_tls_err = m; }

void* qs_context::scratch_get(size_t bytes) {
  if (bytes <= scratch_bytes) return scratch;
  // Grow-only.  Work already queued on the stream may still read the old
  // buffer, so finish it before releasing the memory.
  if (scratch) {
    QS_CUDA(cudaStreamSynchronize(stream));
    QS_CUDA(cudaFree(scratch));
    scratch = nullptr;
    scratch_bytes = 0;
  }
  size_t want = bytes < (1u << 20) ? (1u << 20) : bytes;
  QS_CUDA(cudaMalloc(&scratch, want));
  scratch_bytes = want;
  return scratch;
}

double* qs_context::pinned_get(size_t bytes) {
  if (bytes <= pinned_bytes) return pinned;
  if (pinned) {
    QS_CUDA(cudaStreamSynchronize(stream));
    QS_CUDA(cudaFreeHost(pinned));
    pinned = nullptr;
  }
  size_t want = bytes < 4096 ? 4096 : bytes;
  QS_CUDA(cudaMallocHost((void**)&pinned, want));
  pinned_bytes = want;
  return pinned;
}

static std::atomic<int64_t> g_launches{0};  // every handle of the process

void qs_count_launches(qs_context* h, int64_t delta) {
  h->launches += delta;
  g_launches.fetch_add(delta, std::memory_order_relaxed);
}

void qs_after_launch(qs_context* h, const char* what) {
  h->launches++;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw qs_error(QS_ERR_CUDA, std::string(what) + ": launch failed: " + cudaGetErrorString(e));
}

cudaStream_t qs_upload_stream(qs_context* h) {
  if (!h->upload_stream) QS_CUDA(cudaStreamCreateWithFlags(&h->upload_stream, cudaStreamNonBlocking));
  return h->upload_stream;
}

void qs_pool_keep_at_least(int device, uint64_t keep) {
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess || !pool) return;
  uint64_t cur = 0;
  if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur) == cudaSuccess && cur >= keep) return;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);  // only ever raised
}

extern "C" {

const char* qs_version(void) { return "qsim-b200 0.1.0 (sm_100a)"; }

// The library's stream-ordered allocations (plan programs, batch tables,
// adjoint and noise buffers) come from the device's default memory pool.
// With the pool's default release threshold of 0, everything freed is handed
// back to the driver at each synchronisation and mapped again by the next
// allocation, which costs milliseconds per call; keeping up to 4 GiB cached
// in this process avoids that (a runtime attribute of this process's pool,
// gone when the process exits).  QSIM_POOL_KEEP_BYTES overrides the amount.
static void keep_pool_memory(int device) {
  static std::mutex mu;
  static std::set<int> done;
  std::lock_guard<std::mutex> lk(mu);
  if (!done.insert(device).second) return;
  const char* e = std::getenv("QSIM_POOL_KEEP_BYTES");
  qs_pool_keep_at_least(device, e ? std::strtoull(e, nullptr, 10) : (4ull << 30));
}


int qs_create(int device, qs_handle_t* out) {
  qs_context* h = nullptr;
  QS_API_BEGIN
  QS_CHECK_ARG(out != nullptr, "out is null");
  *out = nullptr;
  int count = 0;
  QS_CUDA(cudaGetDeviceCount(&count));
  QS_CHECK_ARG(device >= 0 && device < count, "device index out of range");
  const qs_device_guard on_device(device);  // the caller's device again on return
  int cur = -1;
  QS_CUDA(cudaGetDevice(&cur));
  if (cur != device) QS_CUDA(cudaSetDevice(device));  // reports why the guard could not select it
  keep_pool_memory(device);
  h = new qs_context();
  h->device = device;
  h->jit_mode = qs_jit_env_mode();
  {
    const char* e = std::getenv("QSIM_BATCH_QUEUE");
    h->batch_queue = (e && e[0] == '1') ? 1 : 0;
    const char* t = std::getenv("QSIM_TC");
    h->tensor_cores = (t && t[0] == '0') ? 0 : 1;
  }
  QS_CUDA(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device));
  QS_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
  h->stream = h->own_stream;
  QS_CUDA(cudaMalloc(&h->dev_status, 256));
  QS_CUDA(cudaMemset(h->dev_status, 0, 256));
  *out = h;
  return QS_OK;
  }
  catch (const qs_error& e) {
    qs_set_tls_error(e.what());
    delete h;
    return e.code;
  }
  catch (const std::exception& e) {
    qs_set_tls_error(e.what());
    delete h;
    return QS_ERR_INVALID;
  }
}

int qs_destroy(qs_handle_t h) {
  if (!h) return QS_OK;
  const qs_device_guard on_device(h->device);
  if (h->own_stream) cudaStreamSynchronize(h->own_stream);
  if (h->stream != h->own_stream) cudaStreamSynchronize(h->stream);
  qs_run_cache_clear(h);
  if (h->upload_stream) {
    cudaStreamSynchronize(h->upload_stream);
    cudaStreamDestroy(h->upload_stream);
  }
  if (h->scratch) cudaFree(h->scratch);
  if (h->dev_status) cudaFree(h->dev_status);
  if (h->pinned) cudaFreeHost(h->pinned);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return QS_OK;
}

int qs_set_stream(qs_handle_t h, void* s) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  // Used verbatim: NULL is the legacy default stream (torch's default).
  h->stream = (cudaStream_t)s;
  QS_API_END(h)
}

void* qs_get_stream(qs_handle_t h) { return h ? (void*)h->stream : nullptr; }

int qs_sync(qs_handle_t h) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CUDA(cudaStreamSynchronize(h->stream));
  QS_API_END(h)
}

const char* qs_last_error(qs_handle_t h) {
  if (h) return h->err.c_str();
  return g_tls_err.c_str();
}

int qs_set_tile_bits(qs_handle_t h, int tile_bits) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(tile_bits == 0 || (tile_bits >= 10 && tile_bits <= 14), "tile_bits must be 0 (auto) or in [10, 14]");
  h->tile_bits = tile_bits;
  QS_API_END(h)
}

int qs_set_block_bits(qs_handle_t h, int bb) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(bb == 0 || (bb >= 2 && bb <= 6), "block_bits must be 0 (auto) or in [2, 6] (6: specialised plans only)");
  h->block_bits = bb;
  QS_API_END(h)
}

int qs_set_jit(qs_handle_t h, int mode, int min_qubits) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(mode >= 0 && mode <= 2, "jit mode must be 0 (off), 1 (large plans) or 2 (every plan)");
  QS_CHECK_ARG(min_qubits >= 0 && min_qubits <= QS_MAX_QUBITS, "min_qubits out of range");
  h->jit_mode = mode;
  if (min_qubits > 0) h->jit_min_qubits = min_qubits;
  QS_API_END(h)
}

int64_t qs_launch_count(qs_handle_t h) { return h ? h->launches : g_launches.load(); }

int qs_device_status(qs_handle_t h, int* code) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(code != nullptr, "code is null");
  uint32_t w = 0;
  QS_CUDA(cudaMemcpyAsync(&w, h->dev_status, sizeof(w), cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaStreamSynchronize(h->stream));
  *code = (int)w;
  if (w) QS_CUDA(cudaMemsetAsync(h->dev_status, 0, sizeof(w), h->stream));
  QS_API_END(h)
}

int qs_set_batch_queue(qs_handle_t h, int on) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(on == 0 || on == 1, "batch mode: 0 one launch per pass level and tile shape, 1 one persistent launch");
  h->batch_queue = on;
  QS_API_END(h)
}

int qs_set_tensor_cores(qs_handle_t h, int on) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(on == 0 || on == 1, "tensor cores: 0 off, 1 on");
  if (h->tensor_cores != on) qs_run_cache_clear(h);  // cached plans were built for the other setting
  h->tensor_cores = on;
  QS_API_END(h)
}

int qs_set_wait_test(qs_handle_t h, int on) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(on >= 0 && on <= 2, "wait test: 0 off, 1 next pipelined pass, 2 next persistent batch launch");
  h->wait_test = on;
  QS_API_END(h)
}

}  // extern "C"
