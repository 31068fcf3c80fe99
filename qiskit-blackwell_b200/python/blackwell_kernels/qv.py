"""Batched Quantum-Volume helpers, call-compatible with the reference's
bwk/python/blackwell_kernels/qv8.py (qv8_simulate, generate_qv8_circuits) and
qv4.py (qv4_simulate_cuda, heavy_output_probability).

Both fixed-width reference kernels (qv8_sim_sm120.cu, qv4_sim_sm120.cu) map
onto the general uneven-width batch engine: each circuit is a list of dense
4x4 ops, planned in FP64 and run as single-CTA shared-memory passes.
"""
from __future__ import annotations

import numpy as np
import torch

from qsim_b200 import engine as E
from qsim_b200.circuit import OP_DTYPE
from qsim_b200.gates import haar_unitary
from qsim_b200._lib import OP_U2


def generate_qv8_circuits(num_circuits, num_layers=8, seed=42, n_qubits=8):
    """Random QV circuits in the reference's layout (qv8.py:76-113): layer
    permutations shared by the batch, Haar U(4) per (circuit, gate).
    Returns gate_matrices [C, G, 4, 4, 2] float32, gate_qubits [C, G, 2] int32, G."""
    rng = np.random.default_rng(seed)
    G = num_layers * (n_qubits // 2)
    perms = [rng.permutation(n_qubits) for _ in range(num_layers)]
    u = haar_unitary(rng, 4, count=num_circuits * G).astype(np.complex64).reshape(num_circuits, G, 4, 4)
    mats = np.stack([u.real, u.imag], axis=-1).astype(np.float32)
    qubits = np.zeros((num_circuits, G, 2), dtype=np.int32)
    g = 0
    for L in range(num_layers):
        for p in range(n_qubits // 2):
            qubits[:, g, 0] = perms[L][2 * p]
            qubits[:, g, 1] = perms[L][2 * p + 1]
            g += 1
    return torch.from_numpy(np.ascontiguousarray(mats)), torch.from_numpy(qubits), G


def _run_fixed(n: int, mats: np.ndarray, qubits: np.ndarray) -> torch.Tensor:
    """mats [C, G, 4, 4] complex, qubits [C, G, 2] (bit 0 = qubits[..., 0])."""
    C, G = qubits.shape[:2]
    ops = np.zeros(C * G, dtype=OP_DTYPE)
    ops["kind"] = OP_U2
    ops["nq"] = 2
    ops["param"] = -1
    ops["q"][:, :2] = qubits.reshape(C * G, 2)
    flat = mats.reshape(C * G, 16).astype(np.complex128)
    ops["m"][:, 0:32:2] = flat.real
    ops["m"][:, 1:32:2] = flat.imag
    widths = np.full(C, n, dtype=np.int32)
    op_off = np.arange(C + 1, dtype=np.int64) * G
    st_off = np.arange(C, dtype=np.int64) << n
    bp = E.BatchPlan(widths, op_off, ops, st_off)
    states = bp.alloc_states()
    bp.execute(states)
    return E.probs_n(states, C << n).reshape(C, 1 << n)


def qv8_simulate(gate_matrices, gate_qubits, num_circuits):
    """probs [C, 256] float32 (qv8.py:192-204); bit 0 of each 4x4 = first qubit."""
    gm = gate_matrices.detach().cpu().numpy() if isinstance(gate_matrices, torch.Tensor) else np.asarray(gate_matrices)
    gq = gate_qubits.detach().cpu().numpy() if isinstance(gate_qubits, torch.Tensor) else np.asarray(gate_qubits)
    gm = gm[:num_circuits]
    gq = gq[:num_circuits].astype(np.int32)
    mats = gm[..., 0] + 1j * gm[..., 1]
    n = int(gq.max()) + 1 if gq.size else 8
    n = max(n, 8)
    return _run_fixed(n, mats, gq)


_PAIRS = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]


def qv4_simulate_cuda(gate_data, pair_ids):
    """probs [C, 16] (qv4.py:53-71); gate_data [C, G, 32] = 16 re + 16 im,
    pair_ids index (0,1),(0,2),(0,3),(1,2),(1,3),(2,3) with bit 0 = lower qubit."""
    gd = gate_data.detach().cpu().numpy() if isinstance(gate_data, torch.Tensor) else np.asarray(gate_data)
    pid = pair_ids.detach().cpu().numpy() if isinstance(pair_ids, torch.Tensor) else np.asarray(pair_ids)
    C, G = pid.shape
    mats = (gd[..., :16] + 1j * gd[..., 16:]).reshape(C, G, 4, 4)
    qubits = np.array(_PAIRS, dtype=np.int32)[pid.astype(np.int64)]
    return _run_fixed(4, mats, qubits)


def heavy_output_probability(probs):
    """Probability mass above the per-circuit median (qv4.py:112-124)."""
    if isinstance(probs, torch.Tensor):
        probs = probs.detach().cpu().numpy()
    med = np.median(probs, axis=1, keepdims=True)
    return (probs * (probs > med)).sum(axis=1)
