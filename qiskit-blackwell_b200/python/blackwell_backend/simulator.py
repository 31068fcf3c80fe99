"""Qiskit-compatible statevector simulator on libqsim.so (B200, sm_100a).

Public surface of the reference's blackwell_backend/simulator.py:
``BlackwellSimulator(device, kernel_path)`` with ``run`` (:555-604),
``run_statevector`` (:606-613), ``run_and_time`` (:615-644) and
``run_hamiltonian`` (:649-723), the same result shapes, counts keys
(hex(basis_index)) and info keys.

What happens underneath differs: a circuit (a qiskit QuantumCircuit, if qiskit
is installed, or a qsim_b200 Circuit) is lowered to libqsim ops, fused in FP64
and cut into tile passes by the C++ planner, and executed with one launch per
pass; the first pass synthesises |0..0> on chip.  Plans are cached per circuit
(simulator.py:500-527 keeps a compile cache the same way).
"""
from __future__ import annotations

import hashlib
import math
import os
import time

import numpy as np
import torch

from qsim_b200 import engine as E
from qsim_b200.circuit import Circuit, from_qiskit, lower


class _Data:
    def __init__(self, counts):
        self.counts = counts

    def to_dict(self):
        return {"counts": self.counts}


class ExperimentResult:
    def __init__(self, shots, success, data, header, metadata=None):
        self.shots = shots
        self.success = success
        self.data = data
        self.header = header
        self.metadata = metadata or {}


class Result:
    """Minimal stand-in for qiskit.result.Result when qiskit is absent."""

    def __init__(self, backend_name, backend_version, qobj_id, job_id, success, results, time_taken):
        self.backend_name = backend_name
        self.backend_version = backend_version
        self.qobj_id = qobj_id
        self.job_id = job_id
        self.success = success
        self.results = results
        self.time_taken = time_taken

    def get_counts(self, experiment=0):
        return dict(self.results[experiment].data.counts)


def _make_result(counts, shots, header, elapsed, metadata=None):
    try:
        from qiskit.result import Result as QResult
        from qiskit.result.models import ExperimentResult as QExp, ExperimentResultData as QData
        exp = QExp(shots=shots, success=True, data=QData(counts=counts), header=header,
                   **({"metadata": metadata} if metadata is not None else {}))
        return QResult(backend_name="blackwell_simulator", backend_version="0.1.0", qobj_id="", job_id="",
                       success=True, results=[exp], time_taken=elapsed)
    except ImportError:
        exp = ExperimentResult(shots, True, _Data(counts), header, metadata)
        return Result("blackwell_simulator", "0.1.0", "", "", True, [exp], elapsed)


def counts_from_samples(samples) -> dict:
    """{hex(index): count} as the reference builds it (simulator.py:579-586).
    A device tensor is histogrammed on the device by libqsim (qs_counts) and
    only the distinct outcomes and their counts are copied back (the
    reference copies every shot and loops over them in Python)."""
    if isinstance(samples, torch.Tensor) and samples.is_cuda:
        keys, cnt = E.counts_arrays(samples.to(torch.int64))
        return dict(zip(map(hex, keys.tolist()), cnt.tolist()))
    vals, cnt = np.unique(np.asarray(samples, dtype=np.int64), return_counts=True)
    return {hex(int(v)): int(c) for v, c in zip(vals, cnt)}


class BlackwellSimulator:
    """Statevector simulator dispatching to libqsim (sm_100a)."""

    def __init__(self, device="cuda", kernel_path=None):
        if kernel_path:
            # A/B hook (simulator.py:43-63): kernel_path names a libqsim.so build
            path = kernel_path if kernel_path.endswith(".so") else os.path.join(kernel_path, "libqsim.so")
            from qsim_b200 import _lib
            if _lib._lib is not None and os.path.abspath(_lib.lib_path()) != os.path.abspath(path):
                raise RuntimeError("a different libqsim.so is already loaded in this process")
            os.environ["QSIM_LIB"] = path
        self.device = device
        self.kernel_path = kernel_path
        self._kernel_label = kernel_path or "libqsim.so"
        self._dev_index = torch.device(device).index if torch.device(device).index is not None else 0
        self._compile_cache = {}
        self._native_1q = {"h", "x", "y", "z", "s", "sdg", "t", "tdg", "rx", "ry", "rz", "p", "u1", "u2", "u3", "u",
                           "id", "sx", "sxdg"}
        self._native_2q = {"cx", "cz", "swap", "cp", "crz", "cu"}
        self._native_mcx = {"ccx"}
        self._native_other = {"measure", "barrier", "reset"}
        # fail loudly now if the library or the GPU is missing
        E._h(self._dev_index)

    # ----------------------------------------------------------- compile --
    def _segments(self, circ: Circuit):
        """Split at measure/reset: list of ('ops', structured array) and
        ('measure', q, c) / ('reset', q)."""
        segs, cur = [], Circuit(circ.num_qubits, circ.num_clbits, circ.name)
        for ins in circ.data:
            if ins.name in ("measure", "reset"):
                if cur.data:
                    segs.append(("ops", lower(cur)))
                    cur = Circuit(circ.num_qubits, circ.num_clbits, circ.name)
                if ins.name == "measure":
                    segs.append(("measure", ins.qubits[0], ins.clbits[0]))
                else:
                    segs.append(("reset", ins.qubits[0]))
            else:
                cur.data.append(ins)
        if cur.data:
            segs.append(("ops", lower(cur)))
        return segs

    def _compile(self, circuit):
        circ = from_qiskit(circuit)
        segs = self._segments(circ)
        key_h = hashlib.sha1()
        key_h.update(str(circ.num_qubits).encode())
        for s in segs:
            key_h.update(s[1].tobytes() if s[0] == "ops" else repr(s).encode())
        key = key_h.hexdigest()
        hit = self._compile_cache.get(key)
        if hit is not None:
            return hit
        compiled = []
        for s in segs:
            if s[0] == "ops":
                compiled.append(("plan", E.Plan(circ.num_qubits, s[1], self._dev_index)) if len(s[1]) else None)
            else:
                compiled.append(s)
        compiled = [c for c in compiled if c is not None]
        entry = (circ.num_qubits, circ.num_clbits, compiled)
        self._compile_cache[key] = entry
        return entry

    # ----------------------------------------------------------- execute --
    def _execute_circuit(self, circuit):
        n, ncl, compiled = self._compile(circuit)
        state = E.empty_state(n, self.device)
        clbits = [0] * ncl
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fresh = True
        for c in compiled:
            if c[0] == "plan":
                if fresh:
                    c[1].execute_from_zero(state)
                else:
                    c[1].execute(state)
            else:
                if fresh:
                    E._h(self._dev_index).call("qs_state_init", E._ptr(state), n)
                outcome = E.measure(state, c[1], torch.rand(1).item())
                if c[0] == "measure":
                    clbits[c[2]] = outcome
                elif outcome == 1:
                    from qsim_b200._lib import OP_MCX
                    import ctypes as C
                    E._h(self._dev_index).call("qs_apply_mcx", E._ptr(state), n, None, 0, int(c[1]))
            fresh = False
        if fresh:
            E._h(self._dev_index).call("qs_state_init", E._ptr(state), n)
        torch.cuda.synchronize()
        return state, clbits, time.perf_counter() - t0

    def _strip_measurements(self, circuit) -> Circuit:
        circ = from_qiskit(circuit)
        out = Circuit(circ.num_qubits, circ.num_clbits, circ.name)
        out.data = [i for i in circ.data if i.name not in ("measure", "reset")]
        return out

    def _run_noisy(self, clean: Circuit, shots: int, seed):
        """Counts of a circuit with noise channels: one trajectory per shot
        (qs_noise_trajectories), trajectories run in chunks of at most 2^26
        amplitudes; trajectory k of the run uses seed + k."""
        from qsim_b200.noise import run_trajectories, sample_trajectories
        base = int(seed) if seed is not None else int(np.random.default_rng().integers(0, 2 ** 62))
        per_chunk = max(1, (1 << 26) >> clean.num_qubits)
        counts = {}
        t0 = time.perf_counter()
        for k0 in range(0, shots, per_chunk):
            k = min(per_chunk, shots - k0)
            states, _ = run_trajectories(clean, k, seed=base + k0, device=self._dev_index, branches=False)
            for key, c in sample_trajectories(states, 1, seed=base + k0).items():
                counts[key] = counts.get(key, 0) + c
        torch.cuda.synchronize()
        return counts, time.perf_counter() - t0

    def run(self, circuit, shots=1024, seed=None):
        """Counts from the pre-measurement statevector (simulator.py:555-604).
        A circuit carrying noise channels (depolarize / amplitude_damp /
        dephase) is sampled as one stochastic trajectory per shot."""
        if seed is not None:
            torch.manual_seed(seed)
            np.random.seed(seed)
        clean = self._strip_measurements(circuit)
        from qsim_b200.circuit import NOISE_OPS
        if any(ins.name in NOISE_OPS for ins in clean.data):
            counts, elapsed = self._run_noisy(clean, int(shots), seed)
            return _make_result(counts, shots, {"name": clean.name, "n_qubits": clean.num_qubits}, elapsed,
                                {"method": "noise trajectories (one per shot)"})
        state, _, elapsed = self._execute_circuit(clean)
        samples = E.sample(state, shots)            # stays on the device
        n = clean.num_qubits
        return _make_result(counts_from_samples(samples), shots, {"name": clean.name, "n_qubits": n}, elapsed)

    def run_statevector(self, circuit):
        """(complex64 numpy statevector, elapsed seconds) (simulator.py:606-613)."""
        state, _, elapsed = self._execute_circuit(circuit)
        return state.cpu().numpy(), elapsed

    def run_statevector_tensor(self, circuit) -> torch.Tensor:
        """The final state as a device tensor (no D2H copy)."""
        return self._execute_circuit(circuit)[0]

    def run_and_time(self, circuit, shots=1024, seed=None, warmup=2, repeats=5):
        if seed is not None:
            torch.manual_seed(seed)
            np.random.seed(seed)
        for _ in range(warmup):
            self._execute_circuit(circuit)
        times = [self._execute_circuit(circuit)[2] for _ in range(repeats)]
        result = self.run(circuit, shots=shots, seed=seed)
        return result, {"times_s": times, "median_s": float(np.median(times)), "min_s": float(np.min(times)),
                        "mean_s": float(np.mean(times))}

    # --------------------------------------------------------- Chebyshev --
    def run_hamiltonian(self, hamiltonian, time_val, initial_state=None, precision=1e-10, shots=None,
                        method="csr"):
        """exp(-iHt)|psi> by Chebyshev expansion (simulator.py:649-723).
        method="csr" builds the CSR as the reference does; method="pauli"
        applies H matrix-free from its Pauli masks."""
        from .chebyshev import chebyshev_evolve, chebyshev_evolve_pauli
        from .hamiltonian import HamiltonianCSR
        from qsim_b200.paulis import PauliSum
        if method == "pauli":
            op = hamiltonian.paulis if isinstance(hamiltonian, HamiltonianCSR) else \
                PauliSum.from_sparse_pauli_op(hamiltonian)
            nq = op.num_qubits
        else:
            op = hamiltonian if isinstance(hamiltonian, HamiltonianCSR) else \
                HamiltonianCSR.from_sparse_pauli_op(hamiltonian, device=self.device)
            nq = op.n_qubits
        if initial_state is None:
            state = E.state_init(nq, self.device)
        else:
            state = initial_state
            if not isinstance(state, torch.Tensor):
                state = torch.as_tensor(np.asarray(state, dtype=np.complex64))
            state = state.to(self.device, torch.complex64).contiguous()
        if method == "pauli":
            result_state, info = chebyshev_evolve_pauli(state, op, time_val, precision=precision)
        else:
            result_state, info = chebyshev_evolve(state, op, time_val, precision=precision)
        hcsr = op if method != "pauli" else None
        if shots is None:
            return result_state.cpu().numpy(), info
        samples = E.sample(result_state, shots)      # histogrammed on the device
        res = _make_result(counts_from_samples(samples), shots,
                           {"name": "chebyshev_evolution", "n_qubits": nq}, info["elapsed_s"], info)
        return res, info
