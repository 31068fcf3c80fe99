"""Seeded synthetic workloads (numpy PCG64 via default_rng).

* ``qv_ops``      — Quantum-Volume-style circuit: each layer a uniformly random
  permutation of the qubits split into adjacent pairs (perm[2p], perm[2p+1]),
  each pair a Haar U(4) with matrix bit 0 on perm[2p] (the layout of
  bwk/python/blackwell_kernels/qv8.py:76-113 and its Haar method, qv8.py:55-73).
* ``layers_ops``  — Haar U(2) on every qubit, CZ brickwork on (2i,2i+1) /
  (2i+1,2i+2) for even / odd layers, a Toffoli on seeded distinct qubits after
  every 5th layer.
* ``qv_batch``    — many QV circuits, widths uniform in [lo, hi], depth = width,
  per-circuit seeds base+i, states packed back to back.
* ``efficient_su2`` / ``random_pauli_observable`` — Ry/Rz layers + CNOT chain
  ansatz with trainable parameters and a random Pauli-sum observable.
* ``serving_hamiltonian`` / ``product_state`` — the Chebyshev requests.
* ``noisy_brickwork`` — RY/RZ on every qubit and CX brickwork per layer, with
  depolarizing, amplitude-damping and dephasing channels after every gate on
  each of its qubits (the noise-trajectory workload).
"""
from __future__ import annotations

import math

import numpy as np

from . import gates as G
from ._lib import OP_MCPHASE, OP_MCX, OP_U1, OP_U2
from .circuit import OP_DTYPE, Circuit
from .paulis import PauliSum


def _set_m(arr, mats):
    flat = mats.reshape(len(arr), -1)
    arr["m"][:, : 2 * flat.shape[1]: 2] = flat.real
    arr["m"][:, 1: 2 * flat.shape[1]: 2] = flat.imag


def qv_ops(n: int, depth: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    npairs = n // 2
    perms = [rng.permutation(n) for _ in range(depth)]
    U = G.haar_unitary(rng, 4, count=depth * npairs)
    ops = np.zeros(depth * npairs, dtype=OP_DTYPE)
    ops["kind"] = OP_U2
    ops["nq"] = 2
    ops["param"] = -1
    k = 0
    for L in range(depth):
        p = perms[L]
        for j in range(npairs):
            ops["q"][k, 0] = p[2 * j]
            ops["q"][k, 1] = p[2 * j + 1]
            k += 1
    _set_m(ops, U)
    return ops


def layers_ops(n: int, layers: int, seed: int, toffoli_every: int = 5) -> np.ndarray:
    rng = np.random.default_rng(seed)
    recs = []
    for L in range(layers):
        U = G.haar_unitary(rng, 2, count=n)
        blk = np.zeros(n, dtype=OP_DTYPE)
        blk["kind"] = OP_U1
        blk["nq"] = 1
        blk["param"] = -1
        blk["q"][:, 0] = np.arange(n)
        _set_m(blk, U)
        recs.append(blk)
        start = 0 if L % 2 == 0 else 1
        pairs = [(a, a + 1) for a in range(start, n - 1, 2)]
        cz = np.zeros(len(pairs), dtype=OP_DTYPE)
        cz["kind"] = OP_MCPHASE
        cz["nq"] = 2
        cz["param"] = -1
        for k, (a, b) in enumerate(pairs):
            cz["q"][k, :2] = (a, b)
        cz["m"][:, 0] = -1.0
        recs.append(cz)
        if toffoli_every and (L + 1) % toffoli_every == 0:
            q = rng.choice(n, 3, replace=False)
            t = np.zeros(1, dtype=OP_DTYPE)
            t["kind"] = OP_MCX
            t["nq"] = 3
            t["param"] = -1
            t["q"][0, :3] = q
            recs.append(t)
    return np.concatenate(recs)


def qv_batch(n_circuits: int, lo: int, hi: int, seed: int):
    """Returns (widths int32[C], op_offsets int64[C+1], ops, state_offsets int64[C])."""
    rng = np.random.default_rng(seed)
    widths = rng.integers(lo, hi + 1, size=n_circuits).astype(np.int32)
    parts = [qv_ops(int(w), int(w), seed * 1_000_003 + i) for i, w in enumerate(widths)]
    sizes = np.array([len(p) for p in parts], dtype=np.int64)
    op_off = np.zeros(n_circuits + 1, dtype=np.int64)
    np.cumsum(sizes, out=op_off[1:])
    ops = np.concatenate(parts) if parts else np.zeros(0, dtype=OP_DTYPE)
    amps = (1 << widths.astype(np.int64))
    st_off = np.zeros(n_circuits, dtype=np.int64)
    if n_circuits > 1:
        np.cumsum(amps[:-1], out=st_off[1:])
    return widths, op_off, ops, st_off


def efficient_su2(n: int, reps: int = 4) -> tuple[Circuit, int]:
    """Ry layer, Rz layer, linear CNOT chain per rep; a final Ry/Rz layer.
    Parameter index: rep r, Ry on q -> 2nr + q, Rz on q -> 2nr + n + q."""
    qc = Circuit(n, name=f"EfficientSU2-{n}")
    for r in range(reps + 1):
        for q in range(n):
            qc.ry(0.0, q, param_index=2 * n * r + q)
        for q in range(n):
            qc.rz(0.0, q, param_index=2 * n * r + n + q)
        if r < reps:
            for q in range(n - 1):
                qc.cx(q, q + 1)
    return qc, 2 * n * (reps + 1)


def random_pauli_observable(n: int, n_terms: int, seed: int, wmin: int = 1, wmax: int = 4) -> PauliSum:
    rng = np.random.default_rng(seed)
    xs, zs, cs = [], [], []
    for _ in range(n_terms):
        w = int(rng.integers(wmin, wmax + 1))
        qs = rng.choice(n, w, replace=False)
        ps = rng.integers(1, 4, size=w)  # 1=X 2=Y 3=Z
        x = z = 0
        for q, p in zip(qs, ps):
            if p in (1, 2):
                x |= 1 << int(q)
            if p in (2, 3):
                z |= 1 << int(q)
        xs.append(x)
        zs.append(z)
        cs.append(float(rng.standard_normal()))
    return PauliSum(xs, zs, cs, n)


def serving_hamiltonian(n: int, seed: int, n_pairs: int = 20) -> PauliSum:
    """sum_ring J_i Z_i Z_{i+1} + sum_i h_i X_i + sum_pairs K (X_a X_b + Y_a Y_b)."""
    rng = np.random.default_rng(seed)
    xs, zs, cs = [], [], []
    J = rng.uniform(-1, 1, size=n)
    h = rng.uniform(-1, 1, size=n)
    for i in range(n):
        a, b = i, (i + 1) % n
        xs.append(0); zs.append((1 << a) | (1 << b)); cs.append(J[i])
    for i in range(n):
        xs.append(1 << i); zs.append(0); cs.append(h[i])
    for _ in range(n_pairs):
        a, b = rng.choice(n, 2, replace=False)
        K = rng.uniform(-0.5, 0.5)
        m = (1 << int(a)) | (1 << int(b))
        xs.append(m); zs.append(0); cs.append(K)      # XX
        xs.append(m); zs.append(m); cs.append(K)      # YY
    return PauliSum(xs, zs, cs, n)


def product_state(n: int, seed: int) -> np.ndarray:
    """Seeded random product state (each qubit Ry(a) Rz(b) |0>), complex128."""
    rng = np.random.default_rng(seed)
    psi = np.ones(1, dtype=np.complex128)
    for _ in range(n):
        a, b = rng.uniform(0, math.pi), rng.uniform(0, 2 * math.pi)
        q = np.array([math.cos(a / 2) * np.exp(-0.5j * b), math.sin(a / 2) * np.exp(0.5j * b)])
        psi = np.kron(q, psi)  # new qubit is the most significant
    return psi


def noisy_brickwork(n: int, layers: int, seed: int, depolarizing: float = 1e-3, amplitude_damping: float = 1e-3,
                    dephasing: float = 1e-3) -> Circuit:
    """Per layer: RY(a) RZ(b) on every qubit (angles uniform in [0, 2pi)),
    then CX on (2i, 2i+1) for even layers and (2i+1, 2i+2) for odd ones; each
    gate followed by the three channels on each qubit it touches."""
    from .noise import add_noise
    rng = np.random.default_rng(seed)
    qc = Circuit(n, name=f"noisy_brickwork_{n}x{layers}")
    for d in range(layers):
        for q in range(n):
            qc.ry(float(rng.uniform(0, 2 * math.pi)), q)
            qc.rz(float(rng.uniform(0, 2 * math.pi)), q)
        for q in range(d % 2, n - 1, 2):
            qc.cx(q, q + 1)
    return add_noise(qc, depolarizing=depolarizing, amplitude_damping=amplitude_damping, dephasing=dephasing)
