"""Sampler / Estimator shaped like Qiskit's V2 primitives, on libqsim.

Qiskit's BackendV2 and primitive classes need qiskit itself (not a
dependency here); these wrappers take the same kinds of inputs — circuits
(native gate set or `unitary`), observables as `SparsePauliOp`, a
`qsim_b200.paulis.PauliSum` or a list of (label, coefficient) pairs — and
return plain Python/numpy results:

    Sampler().run([qc1, qc2], shots=1024)         -> [counts dict, counts dict]
    Estimator().run([(qc, obs), (qc2, obs2)])     -> np.array of <psi|H|psi> (FP64)

Counts are histogrammed on the device (only distinct outcomes are copied
back); expectation values are FP64 fixed-order reductions over the final
state, with no state copied to the host.
"""
from __future__ import annotations

import numpy as np
import torch

from qsim_b200 import engine as E
from qsim_b200.paulis import PauliSum

from .simulator import BlackwellSimulator, counts_from_samples


def _as_pauli_sum(obs, n: int) -> PauliSum:
    if isinstance(obs, PauliSum):
        return obs
    if isinstance(obs, (list, tuple)) and obs and isinstance(obs[0], (list, tuple)):
        return PauliSum.from_list(obs, n)
    return PauliSum.from_sparse_pauli_op(obs)


class Sampler:
    def __init__(self, simulator: BlackwellSimulator | None = None, default_shots: int = 1024):
        self.sim = simulator or BlackwellSimulator()
        self.default_shots = int(default_shots)

    def run(self, circuits, shots: int | None = None, seed: int | None = None) -> list[dict]:
        if not isinstance(circuits, (list, tuple)):
            circuits = [circuits]
        shots = self.default_shots if shots is None else int(shots)
        out = []
        for k, qc in enumerate(circuits):
            if isinstance(qc, tuple):
                qc = qc[0]
            if _is_noisy(qc):   # one trajectory per shot
                out.append(self.sim.run(qc, shots=shots, seed=None if seed is None else int(seed) + k).get_counts())
                continue
            g = None
            if seed is not None:
                g = torch.Generator(device=f"cuda:{self.sim._dev_index}")
                g.manual_seed(int(seed) + k)
            state, _, _ = self.sim._execute_circuit(self.sim._strip_measurements(qc))
            out.append(counts_from_samples(E.sample(state, shots, generator=g)))
        return out


def _is_noisy(qc) -> bool:
    from qsim_b200.circuit import NOISE_OPS, from_qiskit
    return any(ins.name in NOISE_OPS for ins in from_qiskit(qc).data)


class Estimator:
    """trajectories / seed: a circuit with noise channels is estimated as the
    mean of <psi_t|H|psi_t> over that many seeded trajectories (an unbiased
    estimate of Tr(rho H)); noiseless circuits are exact."""

    def __init__(self, simulator: BlackwellSimulator | None = None, trajectories: int = 1024, seed: int = 0):
        self.sim = simulator or BlackwellSimulator()
        self.trajectories = int(trajectories)
        self.seed = int(seed)

    def _noisy_value(self, qc, obs) -> float:
        from qsim_b200.circuit import from_qiskit
        from qsim_b200.noise import run_trajectories
        circ = self.sim._strip_measurements(from_qiskit(qc))
        n = circ.num_qubits
        ps = _as_pauli_sum(obs, n)
        if ps.num_qubits != n:
            raise ValueError(f"observable acts on {ps.num_qubits} qubits, circuit has {n}")
        per_chunk = max(1, (1 << 26) >> n)
        total, done = 0.0, 0
        while done < self.trajectories:
            k = min(per_chunk, self.trajectories - done)
            states, _ = run_trajectories(circ, k, seed=self.seed + done, device=self.sim._dev_index, branches=False)
            total += sum(E.expect_pauli_sum(states[t], ps) for t in range(k))
            done += k
        return total / self.trajectories

    def run(self, pubs) -> np.ndarray:
        """pubs: iterable of (circuit, observable) pairs."""
        vals = []
        for qc, obs in pubs:
            if _is_noisy(qc):
                vals.append(self._noisy_value(qc, obs))
                continue
            state = self.sim.run_statevector_tensor(qc)
            n = state.numel().bit_length() - 1
            ps = _as_pauli_sum(obs, n)
            if ps.num_qubits != n:
                raise ValueError(f"observable acts on {ps.num_qubits} qubits, circuit has {n}")
            vals.append(E.expect_pauli_sum(state, ps))
        return np.asarray(vals, dtype=np.float64)
