// qs_server.cpp — native continuous-batching request server (no reference
// counterpart: the reference runs one circuit per call).
//
// Requests (circuits with shots, adjoint energy+gradient, matrix-free
// Chebyshev evolutions) are submitted from any host thread and get an id.
// A scheduler thread admits queued requests in arrival order against an HBM
// budget (each request counts the device bytes it will hold), drops those
// whose deadline passed while queued, groups admitted circuit requests into
// one batch plan (uneven widths in the same tile-pass launches) and hands
// work items to worker threads.  Every worker owns a libqsim handle on its
// own CUDA stream, so batches, gradients and evolutions run concurrently on
// the device; budget is returned when an item completes, which admits more
// requests.  Worker 0 takes the admitted item of most estimated device work
// (amplitudes x gates for circuits, x passes over the observable for
// gradients, x degree x terms for evolutions), the others the item of least,
// so the large items, which fill the GPU one at a time, run back to back
// while the short ones flow around them instead of queueing behind them.
// Results are identical alone and in a mix: batch plans give the
// same bits as single plans, reductions have a fixed order, and each
// circuit's sampling uniforms come from its own seed.
//
// Failure handling is host-side: too large for the budget -> QS_ERR_BUDGET at
// submit; deadline passed before scheduling -> QS_ERR_TIMEOUT; cancelled
// while queued -> QS_ERR_CANCELLED; an error in an item fails only the
// requests of that item (allocation failures report QS_ERR_NOMEM).
#include "qs_api.h"
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

namespace {

using clock_t_ = std::chrono::steady_clock;

double now_s() {
  return std::chrono::duration<double>(clock_t_::now().time_since_epoch()).count();
}

enum Kind { K_CIRCUIT = 0, K_GRADIENT = 1, K_EVOLUTION = 2 };
enum State { S_QUEUED = 0, S_RUNNING = 1, S_DONE = 2 };

struct Request {
  int64_t id = 0;
  int kind = K_CIRCUIT;
  int n = 0;
  double arrival = 0, deadline_s = 0, done_at = 0;
  size_t need = 0;
  int state = S_QUEUED;
  int status = QS_OK;
  std::string err;
  // circuit
  std::vector<qs_op> ops;
  int64_t shots = 0;
  uint64_t seed = 0;
  std::vector<int64_t> samples;
  // gradient
  int n_params = 0, n_batch = 0;
  std::vector<double> params, energies, grads;
  // Pauli sum (gradient observable / evolution Hamiltonian)
  std::vector<uint64_t> px, pz;
  std::vector<double> pc;
  // evolution
  std::vector<float> psi0, state_out;  // complex64 interleaved
  std::vector<double> cheb;
  int K = 0;
  double scale = 0;
};

using ReqP = std::shared_ptr<Request>;

// Device buffer released when it leaves scope (stream-ordered).
struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  DevBuf(size_t bytes, cudaStream_t stream) : s(stream) {
    if (cudaMallocAsync(&p, bytes, stream) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      throw qs_error(QS_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
  }
  ~DevBuf() {
    if (p) cudaFreeAsync(p, s);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

void check(qs_handle_t h, int rc) {
  if (rc != QS_OK) throw qs_error(rc, qs_last_error(h));
}

}  // namespace

constexpr int64_t kBatchAmps = int64_t(1) << 26;

struct qs_server_s {
  int device = 0;
  int64_t budget = 0, free_bytes = 0;
  int max_batch = 4096;
  std::mutex mu;
  std::condition_variable cv_sched, cv_work, cv_done;
  std::deque<ReqP> queue;                   // waiting for admission
  struct Item {
    std::vector<ReqP> reqs;
    double cost = 0;  // estimated device work
  };
  std::deque<Item> work;                    // admitted items, in admission order
  std::map<int64_t, ReqP> reqs;
  int64_t next_id = 1;
  bool stop = false;
  std::thread scheduler;
  std::vector<std::thread> workers;
  std::vector<double> latencies;
  double t_first = 0, t_last = 0;
  int64_t submitted = 0, completed = 0, failed = 0;

  void finish(const ReqP& r, int status, const std::string& err) {
    // mu held by the caller
    r->status = status;
    r->err = err;
    r->state = S_DONE;
    r->done_at = now_s();
    if (status == QS_OK) {
      ++completed;
      latencies.push_back(r->done_at - r->arrival);
      if (t_first == 0 || r->arrival < t_first) t_first = r->arrival;
      t_last = std::max(t_last, r->done_at);
    } else {
      ++failed;
    }
    cv_done.notify_all();
  }

  // Estimated device work of a request (amplitude updates, arbitrary unit).
  static double cost_of(const Request& r) {
    const double amps = std::ldexp(1.0, r.n);
    if (r.kind == K_CIRCUIT) return amps * (double)(r.ops.size() + 1);
    if (r.kind == K_GRADIENT) return amps * (double)std::max(1, r.n_batch) * (3.0 * r.ops.size() + r.pc.size());
    return amps * (double)std::max(1, r.K) * (0.5 * r.px.size() + 2.0);
  }
  void push_item(std::vector<ReqP>&& reqs) {
    Item it;
    for (const ReqP& r : reqs) it.cost += cost_of(*r);
    it.reqs = std::move(reqs);
    work.push_back(std::move(it));
  }
  // Worker 0: the largest item; the others: the smallest (ties: the oldest).
  std::vector<ReqP> take_item(int worker) {
    auto pick = work.begin();
    for (auto it = work.begin(); it != work.end(); ++it)
      if (worker == 0 ? it->cost > pick->cost : it->cost < pick->cost) pick = it;
    std::vector<ReqP> out = std::move(pick->reqs);
    work.erase(pick);
    return out;
  }

  void schedule_loop() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      cv_sched.wait(lk, [&] { return stop || !queue.empty(); });
      if (stop) return;
      const double t = now_s();
      std::vector<ReqP> circuits;
      int64_t batch_amps = 0;
      std::deque<ReqP> keep;
      while (!queue.empty()) {
        ReqP r = queue.front();
        queue.pop_front();
        if (r->deadline_s > 0 && t - r->arrival > r->deadline_s) {
          finish(r, QS_ERR_TIMEOUT, "deadline passed before the request was scheduled");
          continue;
        }
        if ((int64_t)r->need > free_bytes) {
          keep.push_back(r);
          continue;
        }
        free_bytes -= (int64_t)r->need;
        r->state = S_RUNNING;
        if (r->kind == K_CIRCUIT) {
          // a batch holds at most 2^26 amplitudes (or max_batch circuits), so
          // several batches run on several workers at once; a circuit that
          // large fills the GPU by itself and goes alone
          const int64_t amps = int64_t(1) << r->n;
          if (amps >= kBatchAmps) {
            push_item({r});
            continue;
          }
          if (batch_amps + amps > kBatchAmps || (int)circuits.size() == max_batch) {
            push_item(std::move(circuits));
            circuits.clear();
            batch_amps = 0;
          }
          circuits.push_back(r);
          batch_amps += amps;
        } else {
          push_item({r});
        }
      }
      queue.swap(keep);
      if (!circuits.empty()) push_item(std::move(circuits));
      cv_work.notify_all();
      // with nothing admissible, wait for a completion (or a new request)
      if (!queue.empty()) cv_sched.wait_for(lk, std::chrono::milliseconds(2));
    }
  }

  void worker_loop(int worker) {
    qs_handle_t h = nullptr;
    // This thread's own CUDA calls (buffers, copies) go to the server's device.
    int rc = cudaSetDevice(device) == cudaSuccess ? QS_OK : QS_ERR_CUDA;
    if (rc == QS_OK) rc = qs_create(device, &h);
    for (;;) {
      std::vector<ReqP> item;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || !work.empty(); });
        if (work.empty()) break;  // stop requested and nothing left
        item = take_item(worker);
      }
      int status = QS_OK;
      std::string err;
      try {
        if (rc != QS_OK || !h) throw qs_error(QS_ERR_CUDA, "worker could not create a handle");
        if (item[0]->kind == K_CIRCUIT) run_circuits(h, item);
        else if (item[0]->kind == K_GRADIENT) run_gradient(h, *item[0]);
        else run_evolution(h, *item[0]);
      } catch (const qs_error& e) {
        status = e.code;
        err = e.what();
      } catch (const std::exception& e) {
        status = QS_ERR_INVALID;
        err = e.what();
      }
      if (status != QS_OK && h) qs_sync(h);  // buffers of the failed item are released in order
      std::lock_guard<std::mutex> lk(mu);
      for (const ReqP& r : item) {
        free_bytes += (int64_t)r->need;
        finish(r, status, err);
      }
      cv_sched.notify_all();
    }
    if (h) qs_destroy(h);
  }

  void run_circuits(qs_handle_t h, const std::vector<ReqP>& item) {
    const int nc = (int)item.size();
    std::vector<int32_t> widths(nc);
    std::vector<int64_t> op_off(nc + 1, 0), st_off(nc, 0), shot_off(nc + 1, 0);
    std::vector<qs_op> ops;
    int64_t amps = 0;
    for (int c = 0; c < nc; ++c) {
      const Request& r = *item[c];
      widths[c] = r.n;
      ops.insert(ops.end(), r.ops.begin(), r.ops.end());
      op_off[c + 1] = (int64_t)ops.size();
      st_off[c] = amps;
      amps += int64_t(1) << r.n;
      shot_off[c + 1] = shot_off[c] + r.shots;
    }
    cudaStream_t s = (cudaStream_t)qs_get_stream(h);
    DevBuf states((size_t)std::max<int64_t>(amps, 2) * 8, s);
    qs_batch_plan_t bp = nullptr;
    check(h, qs_batch_plan_create(h, nc, widths.data(), op_off.data(), ops.data(), st_off.data(), &bp));
    std::unique_ptr<qs_batch_plan_s, int (*)(qs_batch_plan_t)> guard(bp, qs_batch_plan_destroy);
    check(h, qs_batch_plan_execute(h, bp, states.p));
    const int64_t total_shots = shot_off[nc];
    std::vector<int64_t> host(total_shots);
    if (total_shots > 0) {
      // every circuit's shots in one batched sampling call (uniforms drawn on
      // the device from each request's seed)
      std::vector<int64_t> shots(nc);
      std::vector<uint64_t> seeds(nc);
      for (int c = 0; c < nc; ++c) {
        shots[c] = item[c]->shots;
        seeds[c] = item[c]->seed;
      }
      DevBuf dout((size_t)total_shots * 8, s);
      check(h, qs_sample_batched(h, states.p, nc, widths.data(), st_off.data(), shots.data(), seeds.data(),
                                 static_cast<int64_t*>(dout.p)));
      QS_CUDA(cudaMemcpyAsync(host.data(), dout.p, (size_t)total_shots * 8, cudaMemcpyDeviceToHost, s));
    }
    check(h, qs_sync(h));  // the plan and buffers outlive the queued work
    for (int c = 0; c < nc; ++c)
      item[c]->samples.assign(host.begin() + shot_off[c], host.begin() + shot_off[c + 1]);
  }

  void run_gradient(qs_handle_t h, Request& r) {
    cudaStream_t s = (cudaStream_t)qs_get_stream(h);
    DevBuf work((size_t)r.n_batch * 3 * ((size_t)8 << r.n), s);
    r.energies.assign(r.n_batch, 0.0);
    r.grads.assign((size_t)r.n_batch * std::max(r.n_params, 1), 0.0);
    check(h, qs_adjoint_gradient(h, r.n, r.ops.data(), (int)r.ops.size(), r.n_params, r.params.data(), r.n_batch,
                                 r.px.data(), r.pz.data(), r.pc.data(), (int)r.pc.size(), work.p, r.energies.data(),
                                 r.grads.data()));
    check(h, qs_sync(h));
  }

  void run_evolution(qs_handle_t h, Request& r) {
    cudaStream_t s = (cudaStream_t)qs_get_stream(h);
    const size_t bytes = (size_t)8 << r.n;
    DevBuf psi(bytes, s), out(bytes, s), work(2 * bytes, s);
    QS_CUDA(cudaMemcpyAsync(psi.p, r.psi0.data(), bytes, cudaMemcpyHostToDevice, s));
    check(h, qs_cheb_evolve_pauli(h, r.n, psi.p, out.p, r.px.data(), r.pz.data(), r.pc.data(), (int)r.pc.size(),
                                  r.cheb.data(), r.K, r.scale, work.p));
    r.state_out.resize((size_t)2 << r.n);
    QS_CUDA(cudaMemcpyAsync(r.state_out.data(), out.p, bytes, cudaMemcpyDeviceToHost, s));
    check(h, qs_sync(h));
  }
};

namespace {

int submit(qs_server_t s, ReqP r, int64_t* id_out) {
  if (r->need > (size_t)s->budget) {
    qs_set_tls_error("request needs " + std::to_string(r->need) + " bytes, more than the server budget of " +
                     std::to_string(s->budget));
    return QS_ERR_BUDGET;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    qs_set_tls_error("server is shutting down");
    return QS_ERR_INVALID;
  }
  r->id = s->next_id++;
  r->arrival = now_s();
  s->reqs[r->id] = r;
  s->queue.push_back(r);
  ++s->submitted;
  *id_out = r->id;
  s->cv_sched.notify_all();
  return QS_OK;
}

ReqP find(qs_server_t s, int64_t id) {
  auto it = s->reqs.find(id);
  return it == s->reqs.end() ? nullptr : it->second;
}

#define SERVER_GUARD(s)                                                  \
  if (!(s)) { qs_set_tls_error("server handle is null"); return QS_ERR_INVALID; }

}  // namespace

extern "C" {

int qs_server_create(int device, int64_t budget_bytes, int n_workers, qs_server_t* out) {
  if (!out || budget_bytes <= 0 || n_workers < 1 || n_workers > 64) {
    qs_set_tls_error("bad server arguments (out, budget > 0, 1..64 workers)");
    return QS_ERR_INVALID;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    qs_set_tls_error("device index out of range");
    return QS_ERR_INVALID;
  }
  // The workers allocate and free their items' buffers (states, block
  // matrices, gradient work) stream-ordered, up to the budget at once; the
  // pool keeps that much mapped, so a synchronisation does not hand it back
  // to the driver only for the next item to map it again.
  qs_pool_keep_at_least(device, (uint64_t)budget_bytes);
  auto* s = new qs_server_s();
  s->device = device;
  s->budget = s->free_bytes = budget_bytes;
  s->scheduler = std::thread([s] { s->schedule_loop(); });
  for (int w = 0; w < n_workers; ++w) s->workers.emplace_back([s, w] { s->worker_loop(w); });
  *out = s;
  return QS_OK;
}

int qs_server_destroy(qs_server_t s) {
  if (!s) return QS_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    // requests still queued are cancelled; admitted items run to completion
    for (const ReqP& r : s->queue) s->finish(r, QS_ERR_CANCELLED, "server shut down");
    s->queue.clear();
  }
  s->cv_sched.notify_all();
  s->cv_work.notify_all();
  if (s->scheduler.joinable()) s->scheduler.join();
  for (auto& w : s->workers)
    if (w.joinable()) w.join();
  delete s;
  return QS_OK;
}

int qs_server_submit_circuit(qs_server_t s, int n_qubits, const qs_op* ops, int n_ops, int64_t shots, uint64_t seed,
                             double deadline_s, int64_t* id_out) {
  SERVER_GUARD(s);
  if (!id_out || n_qubits < 1 || n_qubits > QS_MAX_QUBITS || n_ops < 1 || !ops || shots < 0) {
    qs_set_tls_error("bad circuit request (id_out, 1..34 qubits, >= 1 op, shots >= 0)");
    return QS_ERR_INVALID;
  }
  auto r = std::make_shared<Request>();
  r->kind = K_CIRCUIT;
  r->n = n_qubits;
  r->ops.assign(ops, ops + n_ops);
  r->shots = shots;
  r->seed = seed;
  r->deadline_s = deadline_s;
  r->need = ((size_t)8 << n_qubits) + (size_t)shots * 16;
  return submit(s, r, id_out);
}

int qs_server_submit_gradient(qs_server_t s, int n_qubits, const qs_op* ops, int n_ops, int n_params,
                              const double* params, int n_batch, const uint64_t* x_masks, const uint64_t* z_masks,
                              const double* coefs, int n_terms, double deadline_s, int64_t* id_out) {
  SERVER_GUARD(s);
  if (!id_out || n_qubits < 1 || n_qubits > QS_MAX_QUBITS || n_ops < 1 || !ops || n_params < 0 || n_batch < 1 ||
      (n_params > 0 && !params) || n_terms < 1 || !x_masks || !z_masks || !coefs) {
    qs_set_tls_error("bad gradient request");
    return QS_ERR_INVALID;
  }
  auto r = std::make_shared<Request>();
  r->kind = K_GRADIENT;
  r->n = n_qubits;
  r->ops.assign(ops, ops + n_ops);
  r->n_params = n_params;
  r->n_batch = n_batch;
  if (n_params > 0) r->params.assign(params, params + (size_t)n_params * n_batch);
  r->px.assign(x_masks, x_masks + n_terms);
  r->pz.assign(z_masks, z_masks + n_terms);
  r->pc.assign(coefs, coefs + n_terms);
  r->deadline_s = deadline_s;
  r->need = (size_t)n_batch * 3 * ((size_t)8 << n_qubits);
  return submit(s, r, id_out);
}

int qs_server_submit_evolution(qs_server_t s, int n_qubits, const void* psi0_host, const uint64_t* x_masks,
                               const uint64_t* z_masks, const double* coefs, int n_terms, const double* cheb_coeffs,
                               int K, double scale, double deadline_s, int64_t* id_out) {
  SERVER_GUARD(s);
  if (!id_out || n_qubits < 1 || n_qubits > QS_MAX_QUBITS || !psi0_host || n_terms < 1 || !x_masks || !z_masks ||
      !coefs || !cheb_coeffs || K < 1) {
    qs_set_tls_error("bad evolution request");
    return QS_ERR_INVALID;
  }
  auto r = std::make_shared<Request>();
  r->kind = K_EVOLUTION;
  r->n = n_qubits;
  const float* p = static_cast<const float*>(psi0_host);
  r->psi0.assign(p, p + ((size_t)2 << n_qubits));
  r->px.assign(x_masks, x_masks + n_terms);
  r->pz.assign(z_masks, z_masks + n_terms);
  r->pc.assign(coefs, coefs + n_terms);
  r->cheb.assign(cheb_coeffs, cheb_coeffs + 2 * (size_t)(K + 1));
  r->K = K;
  r->scale = scale;
  r->deadline_s = deadline_s;
  r->need = 4 * ((size_t)8 << n_qubits);
  return submit(s, r, id_out);
}

int qs_server_wait(qs_server_t s, int64_t id, double timeout_s, int* status_out) {
  SERVER_GUARD(s);
  std::unique_lock<std::mutex> lk(s->mu);
  ReqP r = find(s, id);
  if (!r) { qs_set_tls_error("unknown request id"); return QS_ERR_INVALID; }
  const auto pred = [&] { return r->state == S_DONE; };
  if (timeout_s < 0) s->cv_done.wait(lk, pred);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
    qs_set_tls_error("request not finished within the timeout");
    return QS_ERR_TIMEOUT;
  }
  if (status_out) *status_out = r->status;
  return QS_OK;
}

int qs_server_cancel(qs_server_t s, int64_t id) {
  SERVER_GUARD(s);
  std::lock_guard<std::mutex> lk(s->mu);
  ReqP r = find(s, id);
  if (!r) { qs_set_tls_error("unknown request id"); return QS_ERR_INVALID; }
  auto it = std::find(s->queue.begin(), s->queue.end(), r);
  if (it == s->queue.end()) { qs_set_tls_error("request is no longer queued"); return QS_ERR_INVALID; }
  s->queue.erase(it);
  s->finish(r, QS_ERR_CANCELLED, "cancelled before scheduling");
  return QS_OK;
}

const char* qs_server_request_error(qs_server_t s, int64_t id) {
  if (!s) return "server handle is null";
  std::lock_guard<std::mutex> lk(s->mu);
  ReqP r = find(s, id);
  return r ? r->err.c_str() : "unknown request id";
}

int qs_server_result_samples(qs_server_t s, int64_t id, int64_t* out, int64_t n) {
  SERVER_GUARD(s);
  std::lock_guard<std::mutex> lk(s->mu);
  ReqP r = find(s, id);
  if (!r || r->state != S_DONE || r->status != QS_OK || r->kind != K_CIRCUIT || !out ||
      n != (int64_t)r->samples.size()) {
    qs_set_tls_error("no circuit result of that size for this id");
    return QS_ERR_INVALID;
  }
  std::memcpy(out, r->samples.data(), (size_t)n * 8);
  return QS_OK;
}

int qs_server_result_gradient(qs_server_t s, int64_t id, double* energies, double* grads) {
  SERVER_GUARD(s);
  std::lock_guard<std::mutex> lk(s->mu);
  ReqP r = find(s, id);
  if (!r || r->state != S_DONE || r->status != QS_OK || r->kind != K_GRADIENT || !energies || !grads) {
    qs_set_tls_error("no gradient result for this id");
    return QS_ERR_INVALID;
  }
  std::memcpy(energies, r->energies.data(), r->energies.size() * 8);
  for (int b = 0; b < r->n_batch; ++b)
    std::memcpy(grads + (size_t)b * r->n_params, r->grads.data() + (size_t)b * std::max(r->n_params, 1),
                (size_t)r->n_params * 8);
  return QS_OK;
}

int qs_server_result_state(qs_server_t s, int64_t id, void* out_host) {
  SERVER_GUARD(s);
  std::lock_guard<std::mutex> lk(s->mu);
  ReqP r = find(s, id);
  if (!r || r->state != S_DONE || r->status != QS_OK || r->kind != K_EVOLUTION || !out_host) {
    qs_set_tls_error("no evolution result for this id");
    return QS_ERR_INVALID;
  }
  std::memcpy(out_host, r->state_out.data(), r->state_out.size() * sizeof(float));
  return QS_OK;
}

int qs_server_release(qs_server_t s, int64_t id) {
  SERVER_GUARD(s);
  std::lock_guard<std::mutex> lk(s->mu);
  ReqP r = find(s, id);
  if (!r || r->state != S_DONE) { qs_set_tls_error("only finished requests can be released"); return QS_ERR_INVALID; }
  s->reqs.erase(id);
  return QS_OK;
}

int qs_server_stats_get(qs_server_t s, qs_server_stats* out) {
  SERVER_GUARD(s);
  if (!out) { qs_set_tls_error("out is null"); return QS_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> lat = s->latencies;
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double p) {
    if (lat.empty()) return 0.0;
    const double x = p * (double)(lat.size() - 1);
    const size_t i = (size_t)x;
    const double f = x - (double)i;
    return i + 1 < lat.size() ? lat[i] * (1 - f) + lat[i + 1] * f : lat[i];
  };
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->failed = s->failed;
  out->queued = (int64_t)s->queue.size();
  out->p50_ms = pct(0.50) * 1e3;
  out->p99_ms = pct(0.99) * 1e3;
  const double span = s->t_last - s->t_first;
  out->throughput_rps = span > 0 ? (double)s->completed / span : 0.0;
  out->budget_bytes = s->budget;
  out->free_bytes = s->free_bytes;
  return QS_OK;
}

}  // extern "C"
