// qs_tune.cpp — per-width autotuning of the generic tile-pass kernel.
//
// The cost of a plan on the generic kernel depends on the tile width T (how
// many qubits a pass keeps in shared memory: fewer passes vs fewer CTAs per
// SM) and the register-block width R (fusion width 2..5: more work per shared-
// memory round trip vs more registers).  qs_autotune_batch times every
// (T, R) candidate on one sample circuit per distinct width of a batch and
// records the fastest in a process-wide table per device.  Each candidate runs
// as a batch (the batch engine's own launches, tensor-core passes included)
// of up to kTuneSamples distinct circuits of the width, repeated to 2^24
// amplitudes in all, so the choice reflects batch throughput (including the
// per-circuit program switches inside a launch), not the latency of one
// small state on a mostly idle GPU.  Every later plan
// for the generic kernel (batches, single circuits, the adjoint forward pass)
// on that device and width uses it, so a circuit gives the same bits alone
// and in a batch.  Specialised plans keep their own defaults.
#include "qs_api.h"
#include <algorithm>
#include <map>
#include <mutex>

namespace {

struct Shape { int tile_bits, block_bits; };

std::mutex g_tune_mu;
std::map<std::pair<int, int>, Shape>& tune_table() {
  static auto* t = new std::map<std::pair<int, int>, Shape>;  // outlives static destruction
  return *t;
}

constexpr int kTuneMinWidth = 10;
constexpr int kTuneMaxWidth = 24;  // larger states: tuning runs would take seconds

constexpr int kTuneSamples = 8;  // distinct circuits per width in a timing batch

// Device time of one execution of batch B on `scratch` (best of 3 after 1
// warm-up).
float time_batch(qs_context* h, qs_batch_plan_s* B, void* scratch) {
  qs_batch_launch(h, B, scratch);
  cudaEvent_t e0, e1;
  QS_CUDA(cudaEventCreate(&e0));
  QS_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int r = 0; r < 3; ++r) {
    QS_CUDA(cudaEventRecord(e0, h->stream));
    qs_batch_launch(h, B, scratch);
    QS_CUDA(cudaEventRecord(e1, h->stream));
    QS_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    QS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

}  // namespace

void qs_plan_shape(const qs_context* h, int n, bool specialised, int& tile_bits, int& block_bits) {
  tile_bits = h->tile_bits;
  block_bits = h->block_bits;
  if (!specialised && tile_bits == 0 && block_bits == 0) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = tune_table().find({h->device, n});
    if (it != tune_table().end()) {
      tile_bits = it->second.tile_bits;
      block_bits = it->second.block_bits;
    }
  }
  if (tile_bits == 0) tile_bits = 13;
  if (block_bits == 0) block_bits = specialised ? 5 : 4;
}

void qs_circuit_shape(const qs_context* h, int n, const qs_op* ops, int nops, bool specialised, int& tile_bits,
                      int& block_bits) {
  const bool set = specialised || h->tile_bits != 0 || h->block_bits != 0;
  bool tuned = false;
  if (!set) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tuned = tune_table().count({h->device, n}) != 0;
  }
  bool dense = !set && !tuned && qs_tc_enabled(h) && !h->batch_queue && n >= 12 && nops > 0;
  for (int i = 0; dense && i < nops; ++i) dense = ops[i].kind == QS_OP_U2;
  if (dense) {
    tile_bits = 13;
    block_bits = 5;
    return;
  }
  qs_plan_shape(h, n, specialised, tile_bits, block_bits);
}

extern "C" {

int qs_autotune_batch(qs_handle_t h, int nc, const int32_t* widths, const int64_t* op_off, const qs_op* ops) {
  QS_REQUIRE_HANDLE(h);
  void* scratch = nullptr;
  const int saved_jit = h->jit_mode;
  QS_API_BEGIN
  QS_CHECK_ARG(nc >= 0 && (nc == 0 || (widths && op_off && ops)), "null batch descriptor");
  // up to kTuneSamples circuits per distinct width in the tuned range
  std::map<int, std::vector<int>> sample;
  for (int c = 0; c < nc; ++c) {
    QS_CHECK_ARG(widths[c] >= 1 && widths[c] <= QS_MAX_QUBITS, "circuit width out of range");
    if (widths[c] >= kTuneMinWidth && widths[c] <= kTuneMaxWidth && op_off[c + 1] > op_off[c]) {
      auto& v = sample[widths[c]];
      if ((int)v.size() < kTuneSamples) v.push_back(c);
    }
  }
  if (sample.empty()) return QS_OK;
  const int wmax = sample.rbegin()->first;
  constexpr int kFillBits = 24;  // amplitudes per timing run: 2^24 (128 MiB > L2)
  QS_CUDA(cudaMallocAsync(&scratch, (size_t)8 << std::max(wmax, kFillBits), h->stream));
  h->jit_mode = 0;  // time the generic kernel
  for (const auto& kv : sample) {
    const int w = kv.first;
    const std::vector<int>& cs = kv.second;
    // units: the samples repeated (round robin) to fill 2^24 amplitudes
    const uint64_t nunits = w >= kFillBits ? 1ull : std::max<uint64_t>(cs.size(), 1ull << (kFillBits - w));
    std::vector<BatchUnit> units(nunits);
    for (uint64_t u = 0; u < nunits; ++u) units[u] = BatchUnit{(int)(u % cs.size()), u << w, 0, nullptr};
    std::vector<Shape> cands;
    if (w <= 14) {  // one pass: the whole state is the tile
      for (int bb = 2; bb <= std::min(5, w); ++bb) cands.push_back({13, bb});
    } else {
      for (int tb = 12; tb <= 14; ++tb)
        for (int bb = 3; bb <= 5; ++bb) cands.push_back({tb, bb});
    }
    Shape best{13, 4};
    float best_ms = 1e30f;
    for (const Shape& s : cands) {
      std::vector<qs_plan_s> plans(cs.size());
      for (size_t k = 0; k < cs.size(); ++k)
        qs_build_plan(w, ops + op_off[cs[k]], (int)(op_off[cs[k] + 1] - op_off[cs[k]]), s.tile_bits, &plans[k],
                      s.block_bits, false);
      qs_batch_plan_s* B = qs_batch_build_units(h, plans, units, true, 0, false);
      float ms = 1e30f;
      try {
        ms = time_batch(h, B, scratch);
      } catch (...) {
        qs_batch_release(B);
        throw;
      }
      qs_batch_release(B);
      if (ms < best_ms) { best_ms = ms; best = s; }
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_table()[{h->device, w}] = best;
  }
  h->jit_mode = saved_jit;
  QS_CUDA(cudaFreeAsync(scratch, h->stream));
  scratch = nullptr;
  return QS_OK;
  }
  catch (const qs_error& e) {
    h->jit_mode = saved_jit;
    if (scratch) cudaFreeAsync(scratch, h->stream);
    h->err = e.what();
    return e.code;
  }
  catch (const std::exception& e) {
    h->jit_mode = saved_jit;
    if (scratch) cudaFreeAsync(scratch, h->stream);
    h->err = e.what();
    return QS_ERR_INVALID;
  }
}

int qs_autotune_get(int device, int width, int* tile_bits, int* block_bits) {
  if (!tile_bits || !block_bits) { qs_set_tls_error("null output"); return QS_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = tune_table().find({device, width});
  if (it == tune_table().end()) { qs_set_tls_error("width not tuned on this device"); return QS_ERR_INVALID; }
  *tile_bits = it->second.tile_bits;
  *block_bits = it->second.block_bits;
  return QS_OK;
}

int qs_autotune_set(int device, int width, int tile_bits, int block_bits) {
  if (device < 0 || width < 1 || width > 40 || tile_bits < 10 || tile_bits > 14 || block_bits < 2 ||
      block_bits > 5) {
    qs_set_tls_error("autotune entry out of range (device >= 0, width 1..40, tile bits 10..14, block bits 2..5)");
    return QS_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_table()[{device, width}] = Shape{tile_bits, block_bits};
  return QS_OK;
}

int qs_autotune_clear(int device) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto& t = tune_table();
  for (auto it = t.begin(); it != t.end();) {
    if (device < 0 || it->first.first == device) it = t.erase(it); else ++it;
  }
  return QS_OK;
}

}  // extern "C"
