"""Routing of circuits among libqsim's three execution paths.

Same surface as the reference's blackwell_backend/hybrid.py: ``analyze_circuit``
(:51-93), ``RoutingPolicy`` (:98-138) and ``HybridSimulator`` (:143-308) with
``analyze`` / ``run`` / ``run_statevector`` / ``run_both`` / ``route_log`` /
``print_route_summary``.  The reference routes circuits dense in non-native
gates away to Aer GPU, because its own Python per-gate dispatch dominates
there.  Here every gate, ``unitary`` included, goes through the same FP64
planner, so there is nothing to route away from; the routes are instead the
three ways libqsim executes a circuit:

  ``"blackwell"``  the plain path: one fused plan per circuit (cached), one
                   launch per tile pass; lowest latency for one circuit.
  ``"batched"``    one batch plan over many circuits of uneven width, passes
                   of all circuits grouped into shared launches (CUDA graph
                   from the second execution); throughput for many small
                   circuits.
  ``"served"``     the native serving runtime (qs_server_*): requests from
                   any number of callers are admitted against an HBM budget
                   and coalesced into batches by worker threads; returns
                   futures.

Shots on every route are drawn from the same seeded uniforms (splitmix64 of
the seed, as the serving runtime draws them), so a circuit gives identical
counts whichever route runs it.
"""
from __future__ import annotations

import logging
import secrets
import time

import numpy as np
import torch

from qsim_b200 import engine as E
from qsim_b200.circuit import Circuit, from_qiskit, lower

from .simulator import BlackwellSimulator, _make_result, counts_from_samples

logger = logging.getLogger(__name__)

ROUTES = ("blackwell", "batched", "served")

# The gate names the reference counts as native when it computes the
# non-native ratio (hybrid.py:34-48); kept identical so the analysis dicts of
# the two libraries agree for the same circuit.
_REFERENCE_NATIVE = {
    "h", "x", "y", "z", "s", "sdg", "t", "tdg",
    "rx", "ry", "rz", "p", "u1", "u2", "u3", "u",
    "id", "sx", "sxdg",
    "cx", "cz", "swap", "cp", "crz", "cu",
    "ccx",
    "measure", "barrier", "reset",
}

# Stochastic channels (qsim_b200.circuit.NOISE_OPS): only the plain route
# runs them (as one trajectory per shot).
_NOISE_NAMES = {"depolarize", "amplitude_damp", "dephase"}

# Largest amplitude count of one batch plan on the batched route (2^26
# complex64 = 512 MiB of states, the serving runtime's batch cap).
BATCH_AMPS = 1 << 26


def _circuit(circuit) -> Circuit:
    return from_qiskit(circuit)


def analyze_circuit(circuit) -> dict:
    """Gate statistics of a circuit (hybrid.py:51-93): the same keys and
    counting rules as the reference (barriers skipped; a gate is non-native
    when its name is outside the reference's native table)."""
    circ = _circuit(circuit)
    total = native = non_native = n_1q = n_2q = n_mcx = 0
    names = set()
    for ins in circ.data:
        name = ins.name.lower()
        if name == "barrier":
            continue
        total += 1
        names.add(name)
        if name in _REFERENCE_NATIVE:
            native += 1
        else:
            non_native += 1
        k = len(ins.qubits)
        if k == 1:
            n_1q += 1
        elif k == 2:
            n_2q += 1
        else:
            n_mcx += 1
    return {
        "num_qubits": circ.num_qubits,
        "total_gates": total,
        "native_gates": native,
        "non_native_gates": non_native,
        "non_native_ratio": non_native / max(total, 1),
        "n_1q": n_1q,
        "n_2q": n_2q,
        "n_mcx": n_mcx,
        "gate_names": names,
    }


class RoutingPolicy:
    """Chooses a route per circuit (hybrid.py:98-138).

    non_native_threshold: circuits whose non-native ratio exceeds it are
        routed to the batched path when they run as part of a list, even a
        list shorter than batch_min_circuits (the reference sends them to its
        other backend; here they are dense `unitary` circuits such as Quantum
        Volume, which the batch engine's autotuned shapes suit best).
    force_blackwell: circuit names always run on the plain path.
    force_cuquantum: circuit names always sent to the reference's "other"
        backend; here that is the batched path (no Aer in this library).
    force_batched / force_served: circuit names always sent to those routes.
    batch_max_qubits: widest circuit the batched route takes; wider circuits
        fill the GPU alone and gain nothing from sharing launches.
    batch_min_circuits: smallest list routed to the batched path.
    """

    def __init__(self, non_native_threshold=0.3, force_blackwell=None, force_cuquantum=None,
                 force_batched=None, force_served=None, batch_max_qubits=20, batch_min_circuits=2):
        self.non_native_threshold = non_native_threshold
        self.force_blackwell = set(force_blackwell or ())
        self.force_cuquantum = set(force_cuquantum or ())
        self.force_batched = set(force_batched or ())
        self.force_served = set(force_served or ())
        self.batch_max_qubits = int(batch_max_qubits)
        self.batch_min_circuits = int(batch_min_circuits)

    def choose(self, circuit, analysis=None, batch_size=1) -> str:
        """'blackwell', 'batched' or 'served' for `circuit` run in a call
        that carries `batch_size` circuits."""
        name = getattr(circuit, "name", "")
        if name in self.force_blackwell:
            return "blackwell"
        if name in self.force_served:
            return "served"
        if name in self.force_batched or name in self.force_cuquantum:
            return "batched"
        if analysis is None:
            analysis = analyze_circuit(circuit)
        if analysis["gate_names"] & _NOISE_NAMES:
            return "blackwell"          # noise channels run as trajectories on the plain path
        if batch_size > 1 and analysis["num_qubits"] <= self.batch_max_qubits:
            if batch_size >= self.batch_min_circuits or analysis["non_native_ratio"] > self.non_native_threshold:
                return "batched"
        return "blackwell"


class _ServedResult:
    """Future of a served run: result() gives the same Result as run()."""

    def __init__(self, owner, fut, entry, analysis, header, shots, t0):
        self._owner, self._fut, self._entry = owner, fut, entry
        self._analysis, self._header, self._shots, self._t0 = analysis, header, shots, t0
        self._result = None

    def done(self) -> bool:
        return self._fut.done()

    def result(self, timeout=None):
        if self._result is None:
            try:
                samples = self._fut.result(timeout)
            except TimeoutError:
                raise
            except Exception:
                self._entry["success"] = False
                self._owner._route_log.append(self._entry)
                raise
            res = _make_result(counts_from_samples(samples), self._shots, self._header,
                               time.perf_counter() - self._t0)
            self._entry["success"] = True
            self._owner._route_log.append(self._entry)
            self._result = self._owner._attach(res, "served", self._analysis)
        return self._result


class HybridSimulator:
    """Routes circuits to the plain, batched or served path (hybrid.py:143-308).

        sim = HybridSimulator()
        result = sim.run(qc, shots=1024, seed=7)              # policy's choice
        result = sim.run(qc, shots=1024, backend="batched")   # forced route
        results = sim.run([qc1, qc2, ...], shots=1024)        # a list: batched
        fut = sim.submit(qc, shots=1024, seed=7)              # served, async
        choice, analysis = sim.analyze(qc)
    """

    def __init__(self, policy=None, aer_device=None, kernel_path=None, device="cuda",
                 budget_bytes=150 * 10 ** 9, workers=4):
        """aer_device is accepted for signature compatibility and ignored
        (there is no Aer route).  budget_bytes / workers size the serving
        runtime, created on first use of the served route."""
        self.policy = policy or RoutingPolicy()
        self._blackwell = BlackwellSimulator(device=device, kernel_path=kernel_path)
        self._dev = self._blackwell._dev_index
        self._budget, self._workers = int(budget_bytes), int(workers)
        self._server = None
        self._route_log = []

    # ------------------------------------------------------------ helpers --
    def _check_route(self, route):
        if route not in ROUTES:
            raise ValueError(f"unknown route {route!r}: this library routes among {', '.join(ROUTES)}"
                             + (" (there is no Aer/cuQuantum backend)" if route == "cuquantum" else ""))

    def _server_obj(self):
        if self._server is None:
            from qsim_b200.server import NativeServer
            self._server = NativeServer(self._dev, self._budget, self._workers)
        return self._server

    @staticmethod
    def _attach(result, route, analysis):
        # hybrid.py:204-208: routing metadata on the result object
        if not hasattr(result, "metadata"):
            result.metadata = {}
        result.metadata["backend_used"] = route
        result.metadata["analysis"] = analysis
        return result

    @staticmethod
    def _seed(seed):
        return secrets.randbits(63) if seed is None else int(seed)

    def _log_entry(self, circ: Circuit, analysis, route):
        return {
            "circuit_name": circ.name,
            "num_qubits": circ.num_qubits,
            "total_gates": analysis["total_gates"],
            "non_native_ratio": analysis["non_native_ratio"],
            "backend_used": route,
        }

    # ------------------------------------------------------------- public --
    def analyze(self, circuit):
        """(chosen route, analysis dict) without running (hybrid.py:171-175)."""
        analysis = analyze_circuit(circuit)
        return self.policy.choose(circuit, analysis), analysis

    def run(self, circuit, shots=1024, seed=None, backend=None):
        """Counts for one circuit (a Result) or for a list of circuits (a list
        of Results), each Result carrying metadata['backend_used'] and
        metadata['analysis'] (hybrid.py:177-224).  backend forces a route.
        With a list, circuit k is sampled with seed + k."""
        if backend is not None:
            self._check_route(backend)
        if isinstance(circuit, (list, tuple)):
            return self._run_list(list(circuit), shots, seed, backend)
        seed = self._seed(seed)
        circ = _circuit(circuit)
        analysis = analyze_circuit(circ)
        chosen = backend or self.policy.choose(circ, analysis)
        if chosen == "served":
            return self.submit(circ, shots, seed, _analysis=analysis).result()
        if chosen == "batched":
            return self._run_batched([circ], [analysis], shots, seed)[0]
        entry = self._log_entry(circ, analysis, chosen)
        try:
            result = self._run_blackwell(circ, shots, seed)
        except Exception:
            entry["success"] = False
            self._route_log.append(entry)
            raise
        entry["success"] = bool(result.success)
        self._route_log.append(entry)
        logger.info("Routed %s (%dq, %d gates, %.0f%% non-native) -> %s", entry["circuit_name"],
                    entry["num_qubits"], entry["total_gates"], entry["non_native_ratio"] * 100, chosen)
        return self._attach(result, chosen, analysis)

    def submit(self, circuit, shots=1024, seed=None, _analysis=None):
        """Queue one circuit on the serving runtime; returns a future whose
        result() is the same Result run() gives."""
        seed = self._seed(seed)
        circ = _circuit(circuit)
        analysis = _analysis or analyze_circuit(circ)
        clean = self._blackwell._strip_measurements(circ)
        from qsim_b200.server import CircuitRequest
        t0 = time.perf_counter()
        fut = self._server_obj().submit(CircuitRequest(clean.num_qubits, lower(clean), int(shots), seed))
        return _ServedResult(self, fut, self._log_entry(circ, analysis, "served"), analysis,
                             {"name": clean.name, "n_qubits": clean.num_qubits}, int(shots), t0)

    def run_statevector(self, circuit, backend=None):
        """(complex64 numpy statevector, elapsed seconds, route) (hybrid.py:226-236).
        As in the reference, measure/reset collapse the state on the plain
        route; the batched route takes unitary circuits only, and the served
        route returns shots, so it is not a statevector route."""
        circ = _circuit(circuit)
        chosen = backend or self.policy.choose(circ)
        self._check_route(chosen)
        if chosen == "blackwell":
            sv, elapsed = self._blackwell.run_statevector(circ)
            return sv, elapsed, chosen
        if chosen == "batched":
            if any(ins.name in ("measure", "reset") for ins in circ.data):
                raise ValueError("measure/reset collapse the state mid-circuit; the batched route runs "
                                 "unitary circuits only (use the blackwell route)")
            t0 = time.perf_counter()
            states, offs, widths = self._execute_batch([circ])
            sv = states[int(offs[0]): int(offs[0]) + (1 << int(widths[0]))].cpu().numpy()
            return sv, time.perf_counter() - t0, chosen
        raise ValueError("the served route returns shots, not statevectors")

    def run_both(self, circuit, shots=1024, seed=None, routes=("blackwell", "batched")):
        """Run on two routes and compare (hybrid.py:238-265): statevectors,
        fidelity, wall times and speedup of the first over the second."""
        a, b = routes
        sv_a, t_a, _ = self.run_statevector(circuit, backend=a)
        sv_b, t_b, _ = self.run_statevector(circuit, backend=b)
        na = sv_a.astype(np.complex128)                 # compare in FP64
        nb = sv_b.astype(np.complex128)
        na /= np.linalg.norm(na)
        nb /= np.linalg.norm(nb)
        fidelity = float(np.abs(np.vdot(na, nb)) ** 2)
        return {
            f"{a}_sv": sv_a,
            f"{b}_sv": sv_b,
            "fidelity": fidelity,
            f"{a}_time_ms": t_a * 1000,
            f"{b}_time_ms": t_b * 1000,
            "speedup": t_b / max(t_a, 1e-9),
            f"{a}_faster": t_a < t_b,
        }

    @property
    def route_log(self):
        """The routing decisions made so far (hybrid.py:267-270)."""
        return list(self._route_log)

    def print_route_summary(self):
        """Per-route totals and one line per routed circuit (hybrid.py:272-286)."""
        if not self._route_log:
            print("No circuits routed yet.")
            return
        totals = {r: sum(1 for e in self._route_log if e["backend_used"] == r) for r in ROUTES}
        print(f"Routing summary: {len(self._route_log)} circuits")
        print("  " + "  |  ".join(f"{r}: {totals[r]}" for r in ROUTES))
        for e in self._route_log:
            status = "OK" if e["success"] else "FAIL"
            print(f"  {e['circuit_name']:30s} {e['num_qubits']:3d}q "
                  f"{e['total_gates']:4d}g  "
                  f"nn={e['non_native_ratio']:.0%}  "
                  f"-> {e['backend_used']:10s} [{status}]")

    def close(self):
        """Stop the serving runtime, if it was started."""
        if self._server is not None:
            self._server.close()
            self._server = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------- routes ----
    def _run_blackwell(self, circ: Circuit, shots, seed):
        if analyze_circuit(circ)["gate_names"] & _NOISE_NAMES:
            return self._blackwell.run(circ, shots=shots, seed=seed)   # one trajectory per shot
        clean = self._blackwell._strip_measurements(circ)
        state, _, elapsed = self._blackwell._execute_circuit(clean)
        samples = E.sample_seeded(state, shots, seed)
        return _make_result(counts_from_samples(samples), shots, {"name": clean.name, "n_qubits": clean.num_qubits},
                            elapsed)

    def _run_list(self, circuits, shots, seed, backend):
        base = self._seed(seed)
        circs = [_circuit(c) for c in circuits]
        analyses = [analyze_circuit(c) for c in circs]
        routes = [backend or self.policy.choose(c, a, batch_size=len(circs)) for c, a in zip(circs, analyses)]
        results = [None] * len(circs)
        served = []
        batched = [k for k, r in enumerate(routes) if r == "batched"]
        for k, r in enumerate(routes):
            if r == "served":
                served.append((k, self.submit(circs[k], shots, base + k, _analysis=analyses[k])))
        if batched:
            outs = self._run_batched([circs[k] for k in batched], [analyses[k] for k in batched], shots,
                                     [base + k for k in batched])
            for k, res in zip(batched, outs):
                results[k] = res
        for k, r in enumerate(routes):
            if r == "blackwell":
                results[k] = self.run(circs[k], shots, base + k, backend="blackwell")
        for k, fut in served:
            results[k] = fut.result()
        return results

    def _execute_batch(self, cleans):
        """Run stripped circuits as one batch plan: (states, offsets, widths)."""
        widths = np.array([c.num_qubits for c in cleans], dtype=np.int32)
        ops_list = [lower(c) for c in cleans]
        oo = np.zeros(len(cleans) + 1, dtype=np.int64)
        np.cumsum([len(o) for o in ops_list], out=oo[1:])
        ops = np.concatenate(ops_list) if oo[-1] else np.zeros(0, dtype=ops_list[0].dtype)
        amps = np.int64(1) << widths.astype(np.int64)
        so = np.zeros(len(cleans), dtype=np.int64)
        if len(cleans) > 1:
            np.cumsum(amps[:-1], out=so[1:])
        bp = E.BatchPlan(widths, oo, ops, so, self._dev)
        states = bp.alloc_states()
        bp.execute(states)
        return states, so, widths

    def _run_batched(self, circs, analyses, shots, seeds):
        """Batched route: circuits grouped in list order into batch plans of
        at most BATCH_AMPS amplitudes, one plan execution per group."""
        if not isinstance(seeds, (list, tuple)):
            seeds = [int(seeds) + k for k in range(len(circs))]
        cleans = [self._blackwell._strip_measurements(c) for c in circs]
        for c in cleans:
            if (1 << c.num_qubits) > BATCH_AMPS:
                raise ValueError(f"{c.num_qubits}-qubit circuit exceeds the batched route's "
                                 f"{BATCH_AMPS.bit_length() - 1}-qubit limit")
        groups, cur, amps = [], [], 0
        for k, c in enumerate(cleans):
            if cur and amps + (1 << c.num_qubits) > BATCH_AMPS:
                groups.append(cur)
                cur, amps = [], 0
            cur.append(k)
            amps += 1 << c.num_qubits
        if cur:
            groups.append(cur)
        results = [None] * len(circs)
        for g in groups:
            torch.cuda.synchronize(self._dev)
            t0 = time.perf_counter()
            states, so, widths = self._execute_batch([cleans[k] for k in g])
            torch.cuda.synchronize(self._dev)
            elapsed = time.perf_counter() - t0
            samples = [E.sample_seeded(states[int(o): int(o) + (1 << int(w))], shots, seeds[k])
                       for k, o, w in zip(g, so, widths)]
            for k, s in zip(g, samples):
                c = cleans[k]
                res = _make_result(counts_from_samples(s), shots, {"name": c.name, "n_qubits": c.num_qubits},
                                   elapsed)
                entry = self._log_entry(circs[k], analyses[k], "batched")
                entry["success"] = True
                self._route_log.append(entry)
                results[k] = self._attach(res, "batched", analyses[k])
        return results
