// qs_batch.cpp — many independent circuits of uneven width in few launches.
//
// Every circuit is planned on its own (FP64 fusion + tile passes, in
// parallel on the host).  Pass p of every circuit that has one is then
// grouped, by tile size, into one launch of the tile-pass kernel: a circuit
// of <= 14 qubits is a single pass whose tile is the whole state, so it runs
// start to finish in one CTA's shared memory; wider circuits take several
// levels.  All device programs live in one buffer and all item tables in
// another, both built once, so execution issues no host-device copies and can
// be captured in a CUDA graph.
//
// The reference has only fixed-width batches: bwk/csrc/qv8_sim_sm120.cu:58-151
// (8 qubits, one CTA per circuit) and bwk/csrc/batch_sm120.cu:53-279 (one
// launch per gate over [N, 2^n]).
#include "qs_api.h"
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <map>
#include <thread>
#include <tuple>

struct qs_batch_plan_s {
  int device = 0;
  int n_circuits = 0;
  void* d_blob = nullptr;          // all device programs
  void* d_items = nullptr;         // all PassItem tables
  struct Launch {
    int T, R, has2, ncoef;
    size_t item_off;
    int n_items;
    uint64_t total_tiles;
    int threads;
    bool tc;  // tensor-core pass (qs_pass_tc.cu)
  };
  float* d_mats = nullptr;         // block matrices of the tensor-core launches' passes
  std::vector<Launch> launches;
  qs_batch_info info{};
  // CUDA graph of the launch sequence, captured at the second execution on
  // the same states buffer and replayed afterwards
  int executions = 0;
  cudaStream_t stream = nullptr;   // stream of the last upload/execution
  cudaGraphExec_t graph = nullptr;
  void* graph_states = nullptr;
  // one persistent launch (k_pass_queue) instead of `launches`
  bool queue = false;
  uint32_t* d_counters = nullptr;  // 2 + q_items words
  int q_items = 0, q_maxT = 0, q_has2 = 0, q_ncoef = 0;
  uint64_t q_tiles = 0;
  uint32_t q_withhold = 0xffffffffu;  // an item with a dependent (the wait-test hook withholds it)
};

namespace {

void free_bplan(qs_batch_plan_s* b) {
  if (!b) return;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  qs_plan_free_device(b->d_blob, b->stream);
  qs_plan_free_device(b->d_items, b->stream);
  qs_plan_free_device(b->d_counters, b->stream);
  qs_plan_free_device(b->d_mats, b->stream);
  delete b;
}

void plan_all(const qs_context* h, int nc, const int32_t* widths, const int64_t* op_off, const qs_op* ops,
              std::vector<qs_plan_s>& plans) {
  plans.resize(nc);
  std::vector<std::string> errs(nc);
  unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  if (nc < 64) nt = 1;
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; ++t) {
    pool.emplace_back([&, t]() {
      for (int c = (int)t; c < nc; c += (int)nt) {
        try {
          const int64_t b = op_off[c], e = op_off[c + 1];
          if (b < 0 || e < b) throw qs_error(QS_ERR_INVALID, "op_offsets must be non-decreasing");
          int tb = 0, bb = 0;
          qs_circuit_shape(h, widths[c], ops + b, (int)(e - b), false, tb, bb);
          qs_build_plan(widths[c], ops + b, (int)(e - b), tb, &plans[c], bb);
        } catch (const std::exception& ex) {
          errs[c] = ex.what();
        }
      }
    });
  }
  for (auto& th : pool) th.join();
  for (int c = 0; c < nc; ++c)
    if (!errs[c].empty()) throw qs_error(QS_ERR_INVALID, "circuit " + std::to_string(c) + ": " + errs[c]);
}

}  // namespace

// Uploads every plan into one device buffer and groups the (unit, pass)
// items by pass level, then by (T, R, has2), into launches.  Units that
// share a plan share its device program.
qs_batch_plan_s* qs_batch_build_units(qs_context* h, const std::vector<qs_plan_s>& plans,
                                      const std::vector<BatchUnit>& units, bool from_zero, int threads,
                                      bool queue) {
  const int np = (int)plans.size();
  auto* B = new qs_batch_plan_s();
  B->device = h->device;
  B->n_circuits = (int)units.size();
  B->stream = h->stream;
  // The copies go on the upload stream, and the host waits for that stream
  // alone: work already queued on h->stream keeps running meanwhile.  Once
  // the host has seen the copies (and the stream-ordered allocations) done,
  // any stream may use the buffers; they are freed on h->stream.
  cudaStream_t us = nullptr;
  try {
    us = qs_upload_stream(h);
    // concatenate device programs
    std::vector<size_t> boff(np);
    size_t total = 0;
    for (int c = 0; c < np; ++c) {
      boff[c] = total;
      total += (plans[c].blob.size() + 255) & ~size_t(255);
    }
    std::vector<char> blob(total, 0);
    for (int c = 0; c < np; ++c)
      if (!plans[c].blob.empty()) std::memcpy(blob.data() + boff[c], plans[c].blob.data(), plans[c].blob.size());
    if (total) {
      QS_CUDA(cudaMallocAsync(&B->d_blob, total, us));
      QS_CUDA(cudaMemcpyAsync(B->d_blob, blob.data(), total, cudaMemcpyHostToDevice, us));
    }
    for (const BatchUnit& u : units) {
      QS_CHECK_ARG(u.plan >= 0 && u.plan < np, "internal: unit plan index out of range");
      QS_CHECK_ARG(!plans[u.plan].pass_offsets.empty(), "every circuit of a batch needs at least one op");
    }
    int maxp = 0;
    for (auto& p : plans) maxp = std::max(maxp, (int)p.pass_offsets.size());
    std::vector<PassItem> items;
    double bytes = 0, flops = 0;
    if (queue) {
      // one persistent launch: items level by level (larger tiles first
      // within a level), each linked to its state's previous-level item
      B->queue = true;
      std::vector<uint32_t> last(units.size(), 0xffffffffu);
      uint64_t tb = 0;
      for (int L = 0; L < maxp; ++L) {
        std::vector<std::pair<int, size_t>> lvl;  // (T, unit)
        for (size_t u = 0; u < units.size(); ++u)
          if (L < (int)plans[units[u].plan].pass_offsets.size()) lvl.push_back({plans[units[u].plan].pass_T[L], u});
        std::stable_sort(lvl.begin(), lvl.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        for (auto& e : lvl) {
          const BatchUnit& un = units[e.second];
          const qs_plan_s& p = plans[un.plan];
          PassItem it{};
          it.state_off = un.state_off;
          it.pass = reinterpret_cast<const DevPass*>(static_cast<const char*>(B->d_blob) + boff[un.plan] +
                                                     p.pass_offsets[L]);
          it.ntiles = 1ull << (p.n_qubits - p.pass_T[L]);
          it.tile_begin = tb;
          tb += it.ntiles;
          it.flags = (L == 0 && from_zero) ? PI_FROM_ZERO : 0u;
          it.pred = last[e.second];
          if (it.pred != 0xffffffffu && B->q_withhold == 0xffffffffu) B->q_withhold = it.pred;
          it.noise_seed = un.noise_seed;
          it.noise_branch = un.noise_branch;
          last[e.second] = (uint32_t)items.size();
          items.push_back(it);
          B->q_maxT = std::max(B->q_maxT, p.pass_T[L]);
          // 2 (dense 4x4 only) survives only if every item has it
          const int h2 = p.pass_has2[L];
          B->q_has2 = items.size() == 1 ? h2 : (B->q_has2 == h2 ? h2 : ((B->q_has2 | h2) ? 1 : 0));
          B->q_ncoef = std::max(B->q_ncoef, p.pass_ncoef[L]);
          bytes += ((L == 0 && from_zero) ? 8.0 : 16.0) * std::ldexp(1.0, p.n_qubits);
        }
      }
      B->q_items = (int)items.size();
      B->q_tiles = tb;
      if (!items.empty()) QS_CUDA(cudaMallocAsync(&B->d_counters, sizeof(uint32_t) * (2 + items.size()), us));
    }
    // Tensor-core launches: every (plan, level) pass they run gets its block
    // matrices, built on the device after the upload (k_block_mats); an
    // item's mats field holds the pass's first matrix index until the buffer
    // exists.
    std::map<std::pair<int, int>, size_t> mat_first;  // (plan, level) -> matrix index
    std::vector<std::pair<std::pair<int, int>, size_t>> mat_passes;
    size_t n_mats = 0;
    std::vector<size_t> tc_items;
    for (int L = 0; L < (queue ? 0 : maxp); ++L) {
      // key: (T, R, has2); value: items, their plans and the largest coefficient pool
      struct Group {
        std::vector<PassItem> items;
        std::vector<int> plan;
        int ncoef = 0;
      };
      std::map<std::tuple<int, int, int>, Group> groups;
      for (const BatchUnit& u : units) {
        const qs_plan_s& p = plans[u.plan];
        if (L >= (int)p.pass_offsets.size()) continue;
        const int T = p.pass_T[L];
        PassItem it{};
        it.state_off = u.state_off;
        it.pass = reinterpret_cast<const DevPass*>(static_cast<const char*>(B->d_blob) + boff[u.plan] +
                                                   p.pass_offsets[L]);
        it.ntiles = 1ull << (p.n_qubits - T);
        it.flags = (L == 0 && from_zero) ? PI_FROM_ZERO : 0u;
        it.noise_seed = u.noise_seed;
        it.noise_branch = u.noise_branch;
        auto& g = groups[std::make_tuple(T, p.pass_R[L], p.pass_has2[L])];
        g.items.push_back(it);
        g.plan.push_back(u.plan);
        g.ncoef = std::max(g.ncoef, p.pass_ncoef[L]);
        bytes += ((L == 0 && from_zero) ? 8.0 : 16.0) * std::ldexp(1.0, p.n_qubits);
      }
      // larger tiles first: they are the longest-running CTAs
      for (auto g = groups.rbegin(); g != groups.rend(); ++g) {
        qs_batch_plan_s::Launch Lc;
        Lc.T = std::get<0>(g->first);
        Lc.R = std::get<1>(g->first);
        Lc.has2 = std::get<2>(g->first);
        Lc.ncoef = g->second.ncoef;
        Lc.item_off = items.size();
        Lc.n_items = (int)g->second.items.size();
        Lc.tc = qs_tc_pass(h, Lc.T, Lc.R, Lc.has2);
        uint64_t tb = 0;
        for (size_t k = 0; k < g->second.items.size(); ++k) {
          PassItem it = g->second.items[k];
          it.tile_begin = tb;
          tb += it.ntiles;
          if (Lc.tc) {
            const int pl = g->second.plan[k];
            auto key = std::make_pair(pl, L);
            auto f = mat_first.find(key);
            if (f == mat_first.end()) {
              const auto* P = reinterpret_cast<const DevPass*>(plans[pl].blob.data() + plans[pl].pass_offsets[L]);
              f = mat_first.emplace(key, n_mats).first;
              mat_passes.push_back({key, n_mats});
              n_mats += (size_t)P->nblocks;
            }
            it.mats = reinterpret_cast<const float*>((uintptr_t)f->second);
            tc_items.push_back(items.size());
          }
          items.push_back(it);
        }
        Lc.total_tiles = tb;
        Lc.threads = threads;
        B->launches.push_back(Lc);
        if (Lc.tc) ++B->info.n_tc_launches;
      }
    }
    for (const BatchUnit& u : units) flops += plans[u.plan].info.flops;
    std::vector<TcMatJob> jobs;  // host temporary, alive until the synchronisation below
    if (n_mats) {
      constexpr size_t kMat = 8192;  // floats per block matrix (TF32 high part + FP32 remainder)
      QS_CUDA(cudaMallocAsync(&B->d_mats, n_mats * kMat * sizeof(float), us));
      for (size_t k : tc_items)
        items[k].mats = B->d_mats + (size_t)(uintptr_t)items[k].mats * kMat;
      jobs.reserve(n_mats);
      for (const auto& mp : mat_passes) {
        const int pl = mp.first.first, L = mp.first.second;
        const auto* P = reinterpret_cast<const DevPass*>(plans[pl].blob.data() + plans[pl].pass_offsets[L]);
        const auto* dP = reinterpret_cast<const DevPass*>(static_cast<const char*>(B->d_blob) + boff[pl] +
                                                          plans[pl].pass_offsets[L]);
        for (int b = 0; b < P->nblocks; ++b) jobs.push_back(TcMatJob{dP, (uint64_t)b, B->d_mats + (mp.second + b) * kMat});
      }
      void* d_jobs = nullptr;
      QS_CUDA(cudaMallocAsync(&d_jobs, jobs.size() * sizeof(TcMatJob), us));
      QS_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(TcMatJob), cudaMemcpyHostToDevice, us));
      qs_launch_block_mats(h, us, static_cast<const TcMatJob*>(d_jobs), (int)jobs.size());
      QS_CUDA(cudaFreeAsync(d_jobs, us));
    }
    if (!items.empty()) {
      QS_CUDA(cudaMallocAsync(&B->d_items, items.size() * sizeof(PassItem), us));
      QS_CUDA(cudaMemcpyAsync(B->d_items, items.data(), items.size() * sizeof(PassItem), cudaMemcpyHostToDevice,
                              us));
    }
    // blob/items are host temporaries: wait for the copies before they go
    QS_CUDA(cudaStreamSynchronize(us));
    B->info.n_circuits = (int32_t)units.size();
    B->info.n_launches = B->queue ? (B->q_items ? 1 : 0) : (int32_t)B->launches.size();
    B->info.n_items = (int64_t)items.size();
    B->info.max_passes = maxp;
    B->info.bytes_moved = bytes;
    B->info.flops = flops;
  } catch (...) {
    if (us) cudaStreamSynchronize(us);  // no copy may still target the buffers
    free_bplan(B);
    throw;
  }
  return B;
}

// qs_batch_run slices: at most this many, each of at least half this many
// circuits (smaller batches run as one slice).
constexpr int kMaxSlices = 8;
constexpr int kSliceMinCircuits = 256;


static qs_batch_plan_s* build_batch(qs_context* h, int nc, const int32_t* widths, const int64_t* op_off,
                                    const qs_op* ops, const int64_t* state_off) {
  QS_CHECK_ARG(nc >= 0, "n_circuits must be >= 0");
  QS_CHECK_ARG(nc == 0 || (widths && op_off && state_off), "null batch descriptor");
  for (int c = 0; c < nc; ++c) {
    QS_CHECK_ARG(widths[c] >= 1 && widths[c] <= QS_MAX_QUBITS, "circuit width out of range");
    QS_CHECK_ARG(state_off[c] >= 0 && (state_off[c] & 1) == 0, "state offsets must be even and >= 0");
  }
  std::vector<qs_plan_s> plans;
  plan_all(h, nc, widths, op_off, ops, plans);
  std::vector<BatchUnit> units(nc);
  for (int c = 0; c < nc; ++c) units[c] = BatchUnit{c, (uint64_t)state_off[c], 0, nullptr};
  return qs_batch_build_units(h, plans, units, true, 0, h->batch_queue != 0);
}

// Bounded dependency waits: 4 s (a tile takes microseconds; the margin
// covers time slicing with other processes); the wait test uses 50 ms and
// withholds one item that has a dependent.
static void launch_queue_batch(qs_context* h, qs_batch_plan_s* B, void* states) {
  uint32_t withhold = 0xffffffffu;
  uint64_t limit = 4000000000ull;
  if (h->wait_test == 2) {
    withhold = B->q_withhold;
    limit = 50000000ull;
    h->wait_test = 0;
  }
  qs_launch_pass_queue(h, states, static_cast<const PassItem*>(B->d_items), B->q_items, B->q_tiles, B->q_maxT,
                       B->q_has2, B->q_ncoef, B->d_counters, withhold, limit);
}

void qs_batch_launch(qs_context* h, qs_batch_plan_s* B, void* states) {
  B->stream = h->stream;
  if (B->queue) {
    launch_queue_batch(h, B, states);
    return;
  }
  for (const auto& L : B->launches) {
    const PassItem* d = static_cast<const PassItem*>(B->d_items) + L.item_off;
    if (L.tc) qs_launch_pass_tc(h, states, d, L.n_items, L.total_tiles, L.T);
    else qs_launch_pass_items(h, states, d, L.n_items, L.total_tiles, L.T, L.R, L.has2, L.ncoef, L.threads);
  }
}

void qs_batch_release(qs_batch_plan_s* B) { free_bplan(B); }

static void run_batch(qs_context* h, qs_batch_plan_s* B, void* states) {
  if (B->queue) {
    launch_queue_batch(h, B, states);
    return;
  }
  for (const auto& L : B->launches) {
    const PassItem* d = static_cast<const PassItem*>(B->d_items) + L.item_off;
    if (L.tc) qs_launch_pass_tc(h, states, d, L.n_items, L.total_tiles, L.T);
    else qs_launch_pass_items(h, states, d, L.n_items, L.total_tiles, L.T, L.R, L.has2, L.ncoef, L.threads);
  }
}

static bool graphs_enabled() {
  const char* e = std::getenv("QSIM_GRAPHS");
  return !(e && e[0] == '0');
}

// Executes a reusable batch plan.  The first execution launches directly
// (and configures the kernels); the second captures the launch sequence into
// a CUDA graph (on the handle's own stream, since the caller's may be the
// legacy stream, which cannot capture), and every execution on the same
// states buffer then replays it on the caller's stream.  Nothing is captured
// while the caller's stream is itself capturing.
static void run_batch_graphed(qs_context* h, qs_batch_plan_s* B, void* states) {
  ++B->executions;
  B->stream = h->stream;
  if (!graphs_enabled() || B->executions < 2 || B->info.n_launches == 0 || !h->own_stream || h->wait_test) {
    run_batch(h, B, states);
    return;
  }
  if (h->stream) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    QS_CUDA(cudaStreamIsCapturing(h->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
      run_batch(h, B, states);
      return;
    }
  }
  if (!B->graph || B->graph_states != states) {
    if (B->graph) {
      QS_CUDA(cudaGraphExecDestroy(B->graph));
      B->graph = nullptr;
    }
    cudaStream_t caller = h->stream;
    QS_CUDA(cudaStreamBeginCapture(h->own_stream, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t g = nullptr;
    h->stream = h->own_stream;
    try {
      run_batch(h, B, states);
    } catch (...) {
      h->stream = caller;
      cudaStreamEndCapture(h->own_stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    h->stream = caller;
    QS_CUDA(cudaStreamEndCapture(h->own_stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&B->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) throw qs_error(QS_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
    B->graph_states = states;
    qs_count_launches(h, -(int64_t)B->info.n_launches);  // captured, not launched
  }
  QS_CUDA(cudaGraphLaunch(B->graph, h->stream));
  qs_count_launches(h, (int64_t)B->info.n_launches);
}

extern "C" {

int qs_batch_plan_create(qs_handle_t h, int nc, const int32_t* widths, const int64_t* op_off, const qs_op* ops,
                         const int64_t* state_off, qs_batch_plan_t* out) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(out != nullptr, "out is null");
  *out = build_batch(h, nc, widths, op_off, ops, state_off);
  QS_API_END(h)
}

int qs_batch_plan_execute(qs_handle_t h, qs_batch_plan_t B, void* states) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(B != nullptr, "batch plan is null");
  QS_CHECK_ARG(B->n_circuits == 0 || (states && ((uintptr_t)states & 15u) == 0),
               "states must be a 16-byte aligned device pointer");
  QS_CHECK_ARG(B->device == h->device, "batch plan was built for another device");
  run_batch_graphed(h, B, states);
  QS_API_END(h)
}

int qs_batch_plan_info_get(qs_batch_plan_t B, qs_batch_info* info) {
  if (!B || !info) { qs_set_tls_error("null batch plan or info"); return QS_ERR_INVALID; }
  *info = B->info;
  return QS_OK;
}

int qs_batch_plan_destroy(qs_batch_plan_t B) {
  free_bplan(B);
  return QS_OK;
}

// A one-shot batch is planned in slices of about equal op counts, and each
// slice is launched as soon as it is planned: the host plans slice k+1 (and
// copies its programs on the upload stream) while the GPU runs slice k.
static int run_slices(int nc) {
  if (nc < kSliceMinCircuits) return 1;
  return std::min(kMaxSlices, nc / (kSliceMinCircuits / 2));
}

int qs_batch_run(qs_handle_t h, int nc, const int32_t* widths, const int64_t* op_off, const qs_op* ops,
                 void* states, const int64_t* state_off) {
  QS_REQUIRE_HANDLE(h);
  std::vector<qs_batch_plan_s*> Bs;
  auto release = [&]() {
    if (!Bs.empty()) cudaStreamSynchronize(h->stream);  // programs must outlive the launches
    for (auto* B : Bs) free_bplan(B);
    Bs.clear();
  };
  QS_API_BEGIN
  QS_CHECK_ARG(nc >= 0, "n_circuits must be >= 0");
  QS_CHECK_ARG(nc == 0 || (widths && op_off && state_off), "null batch descriptor");
  for (int c = 0; c < nc; ++c) {
    QS_CHECK_ARG(widths[c] >= 1 && widths[c] <= QS_MAX_QUBITS, "circuit width out of range");
    QS_CHECK_ARG(state_off[c] >= 0 && (state_off[c] & 1) == 0, "state offsets must be even and >= 0");
    QS_CHECK_ARG(op_off[c] >= 0 && op_off[c + 1] >= op_off[c], "op_offsets must be non-decreasing");
  }
  const int ns = run_slices(nc);
  const int64_t ops_total = nc ? op_off[nc] - op_off[0] : 0;
  int c0 = 0;
  for (int s = 0; s < ns && c0 < nc; ++s) {
    int c1 = nc;
    if (s + 1 < ns) {  // first circuit past s+1 equal shares of the ops
      const int64_t goal = op_off[0] + ops_total * (s + 1) / ns;
      c1 = c0 + 1;
      while (c1 < nc && op_off[c1] < goal) ++c1;
    }
    Bs.push_back(build_batch(h, c1 - c0, widths + c0, op_off + c0, ops, state_off + c0));
    run_batch(h, Bs.back(), states);
    // the slice's buffers are freed in stream order after its launches, so the
    // next slices reuse the memory (its tensor-core block matrices run to
    // hundreds of MB) instead of every slice's staying allocated to the end
    free_bplan(Bs.back());
    Bs.pop_back();
    c0 = c1;
  }
  release();
  return QS_OK;
  }
  catch (const qs_error& e) {
    h->err = e.what();
    release();
    return e.code;
  }
  catch (const std::exception& e) {
    h->err = e.what();
    release();
    return QS_ERR_INVALID;
  }
}

// Equal-width states back to back: the plan is built once and every pass
// covers all states in one launch (tile ids above 2^(n-T) select the state).
int qs_apply_gates_batched_fused(qs_handle_t h, void* states, int n_states, int n, const float* gates,
                                 const int* targets, int ngates) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(states, n);
  QS_CHECK_ARG(n_states >= 0, "n_states must be >= 0");
  QS_CHECK_ARG(ngates >= 0 && (ngates == 0 || (gates && targets)), "bad gates/targets");
  std::vector<qs_op> ops(ngates);
  for (int g = 0; g < ngates; ++g) {
    qs_op& o = ops[g];
    std::memset(&o, 0, sizeof(o));
    o.kind = QS_OP_U1;
    o.nq = 1;
    o.q[0] = targets[g];
    o.param = -1;
    for (int i = 0; i < 8; ++i) o.m[i] = gates[8 * g + i];
  }
  if (n_states == 0 || ngates == 0) return QS_OK;
  qs_plan_s p;
  int tb = 0, bb = 0;
  qs_plan_shape(h, n, false, tb, bb);
  qs_build_plan(n, ops.data(), ngates, tb, &p, bb);
  qs_plan_upload(h, &p);
  try {
    qs_plan_run(h, &p, states, false, (uint64_t)n_states);
    QS_CUDA(cudaStreamSynchronize(h->stream));
  } catch (...) {
    qs_plan_free_device(p.d_blob, h->stream);
    throw;
  }
  qs_plan_free_device(p.d_blob, h->stream);
  QS_API_END(h)
}

}  // extern "C"
