// qs_counts.cu — measurement counts histogrammed on the device.
//
// The reference builds its counts dictionary with a Python loop over every
// shot after copying all shots to the host (blackwell_backend/simulator.py:
// 579-586).  Here the shots stay on the device: an open-addressing hash table
// (power-of-two size, at least twice the shot count, so at most half full)
// counts them with atomics, a compaction writes the distinct (outcome,
// count) pairs back to back, and the host receives only those pairs.  No
// sort: the caller orders the pairs if it needs an order.
#include "qs_api.h"

namespace {

constexpr int kCThreads = 256;
constexpr unsigned long long kEmpty = ~0ull;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void k_counts_clear(unsigned long long* keys, unsigned int* cnt, uint64_t size, unsigned int* n_out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < size; i += (uint64_t)gridDim.x * blockDim.x) {
    keys[i] = kEmpty;
    cnt[i] = 0u;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = 0u;
}

// Linear probing; the table is at most half full, so every probe sequence
// meets its key or an empty slot within `size` steps.
__global__ void k_counts_insert(const int64_t* __restrict__ shots, uint64_t n, unsigned long long* keys,
                                unsigned int* cnt, uint64_t mask) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long key = (unsigned long long)shots[i];
    uint64_t slot = mix64(key) & mask;
    for (uint64_t probe = 0; probe <= mask; ++probe) {
      const unsigned long long prev = atomicCAS(&keys[slot], kEmpty, key);
      if (prev == kEmpty || prev == key) {
        atomicAdd(&cnt[slot], 1u);
        break;
      }
      slot = (slot + 1) & mask;
    }
  }
}

__global__ void k_counts_compact(const unsigned long long* __restrict__ keys, const unsigned int* __restrict__ cnt,
                                 uint64_t size, int64_t* __restrict__ pairs, unsigned int* n_out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < size; i += (uint64_t)gridDim.x * blockDim.x) {
    if (keys[i] == kEmpty) continue;
    const unsigned int k = atomicAdd(n_out, 1u);
    pairs[2 * k] = (int64_t)keys[i];
    pairs[2 * k + 1] = (int64_t)cnt[i];
  }
}

}  // namespace

extern "C" int qs_counts(qs_handle_t h, const int64_t* shots_dev, int64_t n_shots, int64_t* pairs_host,
                         int64_t capacity, int64_t* n_distinct) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(n_distinct != nullptr, "n_distinct is null");
  QS_CHECK_ARG(n_shots >= 0 && n_shots <= (1ll << 31), "n_shots must be in [0, 2^31]");
  *n_distinct = 0;
  if (n_shots == 0) return QS_OK;
  QS_CHECK_ARG(shots_dev != nullptr && pairs_host != nullptr, "shots/pairs pointer is null");
  uint64_t size = 1024;
  while (size < 2ull * (uint64_t)n_shots) size <<= 1;
  // scratch: keys (8 B) + counts (4 B) per slot, the pair array (16 B per
  // shot at most) and the distinct counter
  const size_t off_cnt = size * 8, off_pairs = off_cnt + size * 4, off_n = off_pairs + (size_t)n_shots * 16;
  char* sc = static_cast<char*>(h->scratch_get(off_n + 64));
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(sc);
  unsigned int* cnt = reinterpret_cast<unsigned int*>(sc + off_cnt);
  int64_t* pairs = reinterpret_cast<int64_t*>(sc + off_pairs);
  unsigned int* n_out = reinterpret_cast<unsigned int*>(sc + off_n);
  const int gs = qs_blocks_for(h, size, kCThreads);
  k_counts_clear<<<gs, kCThreads, 0, h->stream>>>(keys, cnt, size, n_out);
  qs_after_launch(h, "k_counts_clear");
  k_counts_insert<<<qs_blocks_for(h, (uint64_t)n_shots, kCThreads), kCThreads, 0, h->stream>>>(
      shots_dev, (uint64_t)n_shots, keys, cnt, size - 1);
  qs_after_launch(h, "k_counts_insert");
  k_counts_compact<<<gs, kCThreads, 0, h->stream>>>(keys, cnt, size, pairs, n_out);
  qs_after_launch(h, "k_counts_compact");
  unsigned int* pin = reinterpret_cast<unsigned int*>(h->pinned_get(64));
  QS_CUDA(cudaMemcpyAsync(pin, n_out, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaStreamSynchronize(h->stream));
  const int64_t nd = (int64_t)*pin;
  *n_distinct = nd;
  QS_CHECK_ARG(nd <= capacity, "pairs_host holds fewer than the " + std::to_string(nd) + " distinct outcomes");
  QS_CUDA(cudaMemcpyAsync(pairs_host, pairs, (size_t)nd * 16, cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaStreamSynchronize(h->stream));
  QS_API_END(h)
}
