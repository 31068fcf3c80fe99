"""Continuous-batching request server on one GPU.

Requests of three kinds arrive at any time:

* ``CircuitRequest``  — a circuit (qs_op records) + shots -> sampled indices;
* ``GradientRequest`` — parametrised circuit, parameter vector(s) and a Pauli
  observable -> energies and adjoint gradients;
* ``EvolutionRequest``— Pauli-sum Hamiltonian, time, initial state ->
  exp(-iHt)|psi> (Chebyshev, matrix-free Pauli-sum operator).

The scheduler admits queued requests against an HBM budget (default 150 GB,
counting each request's state/workspace bytes), groups the admitted circuit
requests into one batch-plan launch (uneven widths in the same kernels), and
hands work to worker threads.  Each worker owns a libqsim handle bound to its
own CUDA stream, so batches, gradients and evolutions overlap on the device,
and new requests are admitted as soon as earlier ones release memory.

Results do not depend on the mix: the batch engine is bit-identical to a
circuit run alone, every reduction has a fixed order, and each request draws
its sampling uniforms from its own seeded generator.

Failure handling is host-side: a request larger than the budget is rejected
at submit; ``cancel`` drops a queued request; a request whose deadline has
passed before it is scheduled fails with ``DeadlineExceeded``; an exception in
a worker (e.g. a failed allocation) fails only the requests of that batch.
"""
from __future__ import annotations

import ctypes as C
import itertools
import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib


class AdmissionError(RuntimeError):
    pass


class DeadlineExceeded(RuntimeError):
    pass


class Cancelled(RuntimeError):
    pass


_ids = itertools.count()


@dataclass
class CircuitRequest:
    n_qubits: int
    ops: np.ndarray
    shots: int = 1024
    seed: int = 0
    deadline_s: float | None = None

    def bytes_needed(self) -> int:
        return 8 << self.n_qubits


@dataclass
class GradientRequest:
    n_qubits: int
    ops: np.ndarray
    n_params: int
    params: np.ndarray            # [B, n_params]
    observable: object            # PauliSum
    deadline_s: float | None = None

    def bytes_needed(self) -> int:
        b = int(np.asarray(self.params).reshape(-1, max(self.n_params, 1)).shape[0])
        return b * 3 * (8 << self.n_qubits) + (b * self.n_params * 8)


@dataclass
class EvolutionRequest:
    hamiltonian: object           # PauliSum
    t: float
    psi0: np.ndarray | None = None
    precision: float = 1e-6
    deadline_s: float | None = None

    def bytes_needed(self) -> int:
        # psi, out and two recurrence vectors (matrix-free: no CSR)
        return 4 * (8 << self.hamiltonian.num_qubits)


@dataclass(order=True)
class _Job:
    arrival: float
    rid: int
    req: object = field(compare=False)
    fut: Future = field(compare=False)
    need: int = field(compare=False, default=0)
    cancelled: bool = field(compare=False, default=False)


class Server:
    BATCH_AMPS = 1 << 26

    def __init__(self, device: int = 0, budget_bytes: int = 150 * 10 ** 9, workers: int = 4,
                 max_batch_circuits: int = 4096, batch_window_s: float = 0.0005, execute=None):
        """execute(kind, jobs) -> results overrides the GPU executor (host-side
        tests of admission and failure handling use a fake)."""
        self.device = int(device)
        self._execute_override = execute
        self.budget = int(budget_bytes)
        self.free = int(budget_bytes)
        self.max_batch = max_batch_circuits
        self.window = batch_window_s
        self._q: list[_Job] = []
        self._lock = threading.Condition()
        self._work = queue.Queue()
        self._stop = False
        self._jobs = {}
        self.latencies = []
        self.completed = 0
        self.t_first = None
        self.t_last = None
        self._sched = threading.Thread(target=self._schedule, daemon=True)
        self._workers = [threading.Thread(target=self._worker, args=(i,), daemon=True) for i in range(workers)]
        self._sched.start()
        for w in self._workers:
            w.start()

    # ---------------------------------------------------------- client API
    def submit(self, req) -> Future:
        need = req.bytes_needed()
        fut = Future()
        if need > self.budget:
            fut.set_exception(AdmissionError(f"request needs {need} B > budget {self.budget} B"))
            return fut
        job = _Job(time.perf_counter(), next(_ids), req, fut, need)
        fut.rid = job.rid
        with self._lock:
            self._q.append(job)
            self._jobs[job.rid] = job
            self._lock.notify_all()
        return fut

    def cancel(self, fut: Future) -> bool:
        with self._lock:
            job = self._jobs.get(getattr(fut, "rid", -1))
            if job is None or job not in self._q:
                return False
            self._q.remove(job)
            job.cancelled = True
        fut.set_exception(Cancelled("cancelled before scheduling"))
        return True

    def close(self):
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        self._sched.join(5)
        for _ in self._workers:
            self._work.put(None)
        for w in self._workers:
            w.join(30)

    def stats(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        span = (self.t_last - self.t_first) if self.t_first and self.t_last else float("nan")
        return {"completed": self.completed, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "throughput_rps": self.completed / span
                if span and span > 0 else float("nan"), "budget_bytes": self.budget}

    # ---------------------------------------------------------- scheduler
    def _release(self, nbytes: int):
        with self._lock:
            self.free += nbytes
            self._lock.notify_all()

    def _schedule(self):
        while True:
            with self._lock:
                while not self._q and not self._stop:
                    self._lock.wait(0.05)
                if self._stop and not self._q:
                    return
                now = time.perf_counter()
                admitted, keep = [], []
                for job in sorted(self._q):
                    dl = job.req.deadline_s
                    if dl is not None and now - job.arrival > dl:
                        job.fut.set_exception(DeadlineExceeded("deadline passed before scheduling"))
                        continue
                    if job.need <= self.free:
                        self.free -= job.need
                        admitted.append(job)
                    else:
                        keep.append(job)
                self._q = keep
                if not admitted:
                    self._lock.wait(0.002)
                    continue
            # a batch holds at most 2^26 amplitudes (or max_batch circuits) so
            # several batches run on several workers at once; a circuit that
            # large fills the GPU by itself and goes alone
            batch, amps = [], 0
            for j in admitted:
                if not isinstance(j.req, CircuitRequest):
                    continue
                a = 1 << j.req.n_qubits
                if a >= self.BATCH_AMPS:
                    self._work.put(("circuits", [j]))
                    continue
                if batch and (amps + a > self.BATCH_AMPS or len(batch) == self.max_batch):
                    self._work.put(("circuits", batch))
                    batch, amps = [], 0
                batch.append(j)
                amps += a
            if batch:
                self._work.put(("circuits", batch))
            for j in admitted:
                if isinstance(j.req, GradientRequest):
                    self._work.put(("gradient", [j]))
                elif isinstance(j.req, EvolutionRequest):
                    self._work.put(("evolution", [j]))
            if self.window:
                time.sleep(self.window)

    # ------------------------------------------------------------- workers
    def _worker(self, idx: int):
        stream = None
        if self._execute_override is None:
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(device=self.device)
        while True:
            item = self._work.get()
            if item is None:
                return
            kind, jobs = item
            try:
                if self._execute_override is not None:
                    results = self._execute_override(kind, jobs)
                else:
                    with torch.cuda.stream(stream):
                        if kind == "circuits":
                            results = self._run_circuits(jobs)
                        elif kind == "gradient":
                            results = [self._run_gradient(jobs[0])]
                        else:
                            results = [self._run_evolution(jobs[0])]
                        stream.synchronize()
                t = time.perf_counter()
                for j, r in zip(jobs, results):
                    self._done(j, t)
                    j.fut.set_result(r)
            except Exception as e:  # a failed batch fails only its own requests
                for j in jobs:
                    if not j.fut.done():
                        j.fut.set_exception(e)
            finally:
                self._release(sum(j.need for j in jobs))

    def _done(self, job, t):
        self.latencies.append(t - job.arrival)
        self.completed += 1
        if self.t_first is None or job.arrival < self.t_first:
            self.t_first = job.arrival
        self.t_last = t

    def _run_circuits(self, jobs):
        from . import engine as E
        widths = np.array([j.req.n_qubits for j in jobs], dtype=np.int32)
        sizes = np.array([len(j.req.ops) for j in jobs], dtype=np.int64)
        oo = np.zeros(len(jobs) + 1, dtype=np.int64)
        np.cumsum(sizes, out=oo[1:])
        ops = np.concatenate([j.req.ops for j in jobs])
        amps = 1 << widths.astype(np.int64)
        so = np.zeros(len(jobs), dtype=np.int64)
        if len(jobs) > 1:
            np.cumsum(amps[:-1], out=so[1:])
        bp = E.BatchPlan(widths, oo, ops, so, self.device)
        states = bp.alloc_states()
        bp.execute(states)
        # all samples are queued on the worker's stream, then copied back in
        # one transfer (one synchronisation per batch, not per circuit)
        dev_out = []
        for j, off, w in zip(jobs, so, widths):
            g = torch.Generator(device=f"cuda:{self.device}")
            g.manual_seed(int(j.req.seed))
            st = states[int(off): int(off) + (1 << int(w))]
            dev_out.append(E.sample(st, j.req.shots, generator=g))
        host = torch.cat(dev_out).cpu().numpy() if dev_out else np.zeros(0, dtype=np.int64)
        out, k = [], 0
        for j in jobs:
            out.append(host[k: k + j.req.shots])
            k += j.req.shots
        del bp
        return out

    def _run_gradient(self, job):
        from . import engine as E
        r = job.req
        e, g = E.adjoint_gradient(r.n_qubits, r.ops, r.n_params, np.asarray(r.params), r.observable, self.device)
        return e, g

    def _run_evolution(self, job):
        from blackwell_backend.chebyshev import chebyshev_evolve_pauli
        r = job.req
        n = r.hamiltonian.num_qubits
        if r.psi0 is None:
            from . import engine as E
            psi = E.state_init(n, f"cuda:{self.device}")
        else:
            psi = torch.as_tensor(np.asarray(r.psi0, dtype=np.complex64)).to(f"cuda:{self.device}")
        out, info = chebyshev_evolve_pauli(psi, r.hamiltonian, r.t, precision=r.precision)
        return out.cpu().numpy(), info


# ---------------------------------------------------------------- native
class _NativeFuture:
    """Result handle of a NativeServer request."""

    def __init__(self, srv, rid: int, req):
        self._srv, self.rid, self._req = srv, rid, req
        self._value = None
        self._done = False

    def done(self) -> bool:
        st = C.c_int(0)
        return self._srv.L.qs_server_wait(self._srv.ptr, self.rid, 0.0, C.byref(st)) == 0

    def result(self, timeout: float | None = None):
        if self._done:
            return self._value
        L, p = self._srv.L, self._srv.ptr
        st = C.c_int(0)
        rc = L.qs_server_wait(p, self.rid, -1.0 if timeout is None else float(timeout), C.byref(st))
        if rc != 0:
            raise TimeoutError(f"request {self.rid} not finished within {timeout} s")
        if st.value != 0:
            msg = (L.qs_server_request_error(p, self.rid) or b"").decode()
            L.qs_server_release(p, self.rid)
            self._done = True
            if st.value == 5:
                raise AdmissionError(msg)
            if st.value == 4:
                raise DeadlineExceeded(msg)
            if st.value == 6:
                raise Cancelled(msg)
            raise RuntimeError(f"request failed ({st.value}): {msg}")
        r = self._req
        if isinstance(r, CircuitRequest):
            out = np.empty(int(r.shots), dtype=np.int64)
            _lib.check(L.qs_server_result_samples(p, self.rid, out.ctypes.data_as(C.c_void_p), int(r.shots)))
            self._value = out
        elif isinstance(r, GradientRequest):
            P = np.asarray(r.params).reshape(-1, max(r.n_params, 1))
            e = np.zeros(P.shape[0])
            g = np.zeros((P.shape[0], r.n_params))
            _lib.check(L.qs_server_result_gradient(p, self.rid, e.ctypes.data_as(C.c_void_p),
                                                   g.ctypes.data_as(C.c_void_p)))
            self._value = (e, g)
        else:
            out = np.empty(1 << r.hamiltonian.num_qubits, dtype=np.complex64)
            _lib.check(L.qs_server_result_state(p, self.rid, out.ctypes.data_as(C.c_void_p)))
            self._value = (out, self._info)
        L.qs_server_release(p, self.rid)
        self._done = True
        return self._value


class NativeServer:
    """The same request types served by the C++ runtime (qs_server_* in the C
    ABI): scheduling, admission, batching and the worker threads are native;
    this class only marshals requests and results.  Sampling uniforms come
    from each circuit request's seed (splitmix64), so results are identical
    alone and in a mix (they differ from the Python Server's torch RNG)."""

    def __init__(self, device: int = 0, budget_bytes: int = 150 * 10 ** 9, workers: int = 4):
        self.L = _lib.load()
        out = C.c_void_p()
        _lib.check(self.L.qs_server_create(int(device), int(budget_bytes), int(workers), C.byref(out)))
        self.ptr = out

    def submit(self, req) -> _NativeFuture:
        L, p = self.L, self.ptr
        rid = C.c_int64(0)
        dl = float(req.deadline_s or 0.0)
        if isinstance(req, CircuitRequest):
            ops = np.ascontiguousarray(req.ops)
            rc = L.qs_server_submit_circuit(p, int(req.n_qubits), ops.ctypes.data_as(C.POINTER(_lib.QsOp)),
                                            int(len(ops)), int(req.shots), int(req.seed) & (2 ** 64 - 1), dl,
                                            C.byref(rid))
            fut = _NativeFuture(self, rid.value, req)
        elif isinstance(req, GradientRequest):
            ops = np.ascontiguousarray(req.ops)
            P = np.ascontiguousarray(np.asarray(req.params, dtype=np.float64).reshape(-1, max(req.n_params, 1)))
            x = np.ascontiguousarray(req.observable.x, dtype=np.uint64)
            z = np.ascontiguousarray(req.observable.z, dtype=np.uint64)
            c = np.ascontiguousarray(req.observable.real_coefs(), dtype=np.float64)
            rc = L.qs_server_submit_gradient(p, int(req.n_qubits), ops.ctypes.data_as(C.POINTER(_lib.QsOp)),
                                             int(len(ops)), int(req.n_params), P.ctypes.data_as(C.c_void_p),
                                             int(P.shape[0]), x.ctypes.data_as(C.c_void_p),
                                             z.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p),
                                             int(len(c)), dl, C.byref(rid))
            fut = _NativeFuture(self, rid.value, req)
        else:
            from blackwell_backend.chebyshev import chebyshev_coefficients
            H = req.hamiltonian
            n = H.num_qubits
            psi = np.ascontiguousarray(np.asarray(req.psi0, dtype=np.complex64) if req.psi0 is not None
                                       else np.eye(1, 1 << n, dtype=np.complex64)[0])
            bound = H.spectral_bound()
            coeffs, K, tail = chebyshev_coefficients(req.t, bound, req.precision)
            cbuf = np.ascontiguousarray(np.stack([coeffs.real, coeffs.imag], axis=-1).reshape(-1), dtype=np.float64)
            x = np.ascontiguousarray(H.x, dtype=np.uint64)
            z = np.ascontiguousarray(H.z, dtype=np.uint64)
            c = np.ascontiguousarray(H.real_coefs(), dtype=np.float64)
            rc = L.qs_server_submit_evolution(p, n, psi.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p),
                                              z.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p),
                                              int(len(c)), cbuf.ctypes.data_as(C.c_void_p), int(K),
                                              float(1.0 / bound), dl, C.byref(rid))
            fut = _NativeFuture(self, rid.value, req)
            fut._info = {"engine": "chebyshev-b200-pauli", "chebyshev_degree": K, "spectral_bound": bound,
                         "truncation_error_bound": tail}
        if rc != 0:
            msg = (L.qs_last_error(None) or b"").decode()
            f = Future()
            f.set_exception(AdmissionError(msg) if rc == 5 else RuntimeError(f"submit failed ({rc}): {msg}"))
            return f
        return fut

    def cancel(self, fut) -> bool:
        return isinstance(fut, _NativeFuture) and self.L.qs_server_cancel(self.ptr, fut.rid) == 0

    def stats(self) -> dict:
        s = _lib.QsServerStats()
        _lib.check(self.L.qs_server_stats_get(self.ptr, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _lib.QsServerStats._fields_}

    def close(self):
        if getattr(self, "ptr", None):
            self.L.qs_server_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
