"""FP64 CPU oracle — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module, as the checker (or the timed CPU baseline); the product never
does.  Two independent restatements of the reference's algorithm are kept:

* ``C``: oracle/sv64.c (FP64, OpenMP) — consumes the qs_op records of
  include/qsim.h; used for large states and the CPU baseline.
* ``numpy``: ``apply_ops_np`` below, an einsum/tensor restatement for small n,
  cross-checked against the C oracle in the tests.

Semantics followed (reference DarrellThomas/qiskit-blackwell):
  1Q pairs / 2Q index order        bwk/csrc/apply_gate_sm120.cu:10-14, apply_gate2q_sm120.cu:11-20
  controls (insert zeros + mask)   bwk/csrc/apply_mcgate_sm120.cu:62-98
  diagonals                        bwk/csrc/apply_diagonal_sm120.cu:43-105
  sampling: smallest i, cdf[i]>=u  bwk/csrc/sample_sm120.cu:61-68 (clamped to N-1)
  measurement: outcome 0 iff u<p0  bwk/csrc/measure_sm120.cu:88-106
  Pauli Z / X,Y expectations       bwk/csrc/expectation_sm120.cu:45-163
  Chebyshev: dense expm reference  tests/ab_test.py:424-466 (scipy.linalg.expm)
Parity pins: tests/golden/ fixtures made from the reference's own Python
(qv8_simulate_ref, qv4_simulate_numpy, chebyshev_coefficients) by
tests/golden/make_golden.py, plus the analytic pins of tests/stress_test.py.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import build_oracle  # noqa: E402

_lib = None

# qs_op layout (include/qsim.h)
OP_DTYPE = np.dtype([("kind", "<i4"), ("nq", "<i4"), ("q", "<i4", (8,)), ("param", "<i4"), ("flags", "<i4"),
                     ("m", "<f8", (32,))])
U1, U2, DIAG1, DIAG2, MCU1, MCU2, MCX, MCSWAP, MCPHASE, Y, RX, RY, RZ = range(1, 14)


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.build()
        L = C.CDLL(path)
        L.sv64_init.argtypes = [C.c_void_p, C.c_int]
        L.sv64_apply_ops.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.sv64_apply_ops.restype = C.c_int
        L.sv64_fidelity_c64.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.sv64_fidelity_c64.restype = C.c_double
        L.sv64_max_abs_err_c64.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.sv64_max_abs_err_c64.restype = C.c_double
        L.sv64_expect_pauli.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.sv64_expect_pauli.restype = C.c_double
        _lib = L
    return _lib


def _ops(ops):
    ops = np.ascontiguousarray(ops)
    if ops.dtype.itemsize != 304:
        raise ValueError("ops must be qs_op records")
    return ops


def simulate(n: int, ops, psi0: np.ndarray | None = None) -> np.ndarray:
    """FP64 final state U|psi0> (|0..0> by default) via the C oracle."""
    ops = _ops(ops)
    if psi0 is None:
        psi = np.empty(1 << n, dtype=np.complex128)
        lib().sv64_init(psi.ctypes.data, n)
    else:
        psi = np.array(psi0, dtype=np.complex128, copy=True)
    rc = lib().sv64_apply_ops(psi.ctypes.data, n, ops.ctypes.data, len(ops))
    if rc != 0:
        raise ValueError("oracle: unsupported op kind")
    return psi


def fidelity(a64c: np.ndarray, b: np.ndarray) -> float:
    """|<a|b>|^2 / (|a|^2|b|^2); a complex64, b complex128."""
    a = np.ascontiguousarray(a64c, dtype=np.complex64)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    n = int(a.size).bit_length() - 1
    return lib().sv64_fidelity_c64(a.ctypes.data, b.ctypes.data, n)


def max_abs_err(a64c: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a64c, dtype=np.complex64)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    n = int(a.size).bit_length() - 1
    return lib().sv64_max_abs_err_c64(a.ctypes.data, b.ctypes.data, n)


# ------------------------------------------------------- numpy restatement
def _mat(rec, k):
    m = rec["m"]
    return np.array([m[2 * i] + 1j * m[2 * i + 1] for i in range(k)], dtype=np.complex128)


def _apply_k(psi, n, targets, G, controls=()):
    """Apply a 2^k x 2^k matrix G (index bit j = targets[j]) under controls,
    with tensor reshapes (axis of qubit q is n-1-q in C order)."""
    t = psi.reshape((2,) * n)
    k = len(targets)
    sl = [slice(None)] * n
    for c in controls:
        sl[n - 1 - c] = 1
    sub = t[tuple(sl)]
    # remaining axes: qubits not in controls, descending order
    rem = [q for q in range(n - 1, -1, -1) if q not in controls]
    ax = [rem.index(q) for q in targets]  # axis of target j
    Gt = G.reshape((2,) * (2 * k))        # out bits (k-1..0), in bits (k-1..0)
    # matrix index bit j = targets[j] -> tensor axis order (targets[k-1], ..., targets[0])
    in_axes = [ax[j] for j in range(k - 1, -1, -1)]
    moved = np.moveaxis(sub, in_axes, list(range(k)))
    shp = moved.shape
    flat = moved.reshape(2 ** k, -1)
    out = (G @ flat).reshape(shp)
    sub[...] = np.moveaxis(out, list(range(k)), in_axes)
    t[tuple(sl)] = sub
    return t.reshape(-1)


def apply_ops_np(psi: np.ndarray, n: int, ops) -> np.ndarray:
    """Independent numpy restatement (small n)."""
    psi = np.array(psi, dtype=np.complex128, copy=True)
    idx = np.arange(1 << n, dtype=np.int64)
    for r in _ops(ops):
        kind, nq = int(r["kind"]), int(r["nq"])
        q = [int(x) for x in r["q"][:nq]]
        if kind == U1:
            psi = _apply_k(psi, n, [q[0]], _mat(r, 4).reshape(2, 2))
        elif kind == MCU1:
            psi = _apply_k(psi, n, [q[-1]], _mat(r, 4).reshape(2, 2), q[:-1])
        elif kind == MCX:
            psi = _apply_k(psi, n, [q[-1]], np.array([[0, 1], [1, 0]], dtype=complex), q[:-1])
        elif kind == Y:
            psi = _apply_k(psi, n, [q[0]], np.array([[0, -1j], [1j, 0]]))
        elif kind in (RX, RY, RZ):
            th = float(r["m"][0])
            c, s = math.cos(th / 2), math.sin(th / 2)
            G = {RX: [[c, -1j * s], [-1j * s, c]], RY: [[c, -s], [s, c]],
                 RZ: [[np.exp(-0.5j * th), 0], [0, np.exp(0.5j * th)]]}[kind]
            psi = _apply_k(psi, n, [q[0]], np.array(G, dtype=complex))
        elif kind in (U2, MCU2):
            psi = _apply_k(psi, n, q[-2:], _mat(r, 16).reshape(4, 4), q[:-2])
        elif kind == MCSWAP:
            psi = _apply_k(psi, n, q[-2:], np.eye(4, dtype=complex)[[0, 2, 1, 3]], q[:-2])
        elif kind == MCPHASE:
            m = 0
            for x in q:
                m |= 1 << x
            sel = (idx & m) == m
            psi[sel] *= _mat(r, 1)[0]
        elif kind in (DIAG1, DIAG2):
            k = 1 if kind == DIAG1 else 2
            d = _mat(r, 1 << k)
            sel = np.zeros_like(idx)
            for j in range(k):
                sel |= ((idx >> q[j]) & 1) << j
            psi *= d[sel]
        else:
            raise ValueError(f"unsupported op kind {kind}")
    return psi


def zero_state(n: int) -> np.ndarray:
    psi = np.zeros(1 << n, dtype=np.complex128)
    psi[0] = 1
    return psi


# --------------------------------------------------------------- reductions
def sample_indices(psi: np.ndarray, u: np.ndarray) -> np.ndarray:
    """smallest i with cdf[i] >= u (FP64 cdf), clamped to N-1."""
    cdf = np.cumsum(np.abs(psi) ** 2)
    out = np.searchsorted(cdf, u, side="left")
    return np.minimum(out, psi.size - 1)


def pauli_expectation_c(psi: np.ndarray, x, z, c) -> float:
    """pauli_expectation by the C oracle (FP64, OpenMP): for 20+ qubits and
    hundreds of terms, where the numpy loop takes seconds per call."""
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    n = int(psi.size).bit_length() - 1
    x = np.ascontiguousarray(x, dtype=np.uint64)
    z = np.ascontiguousarray(z, dtype=np.uint64)
    c = np.ascontiguousarray(c, dtype=np.float64)
    return float(lib().sv64_expect_pauli(psi.ctypes.data, n, x.ctypes.data, z.ctypes.data, c.ctypes.data,
                                         int(c.size)))


def pauli_expectation(psi: np.ndarray, x, z, c) -> float:
    """sum_t c_t <psi|P_t|psi>, P = i^{|x&z|} X^x Z^z."""
    idx = np.arange(psi.size, dtype=np.uint64)
    tot = 0.0
    for xm, zm, cm in zip(x, z, c):
        xm, zm = np.uint64(xm), np.uint64(zm)
        ny = bin(int(xm & zm)).count("1")
        j = idx ^ xm
        sgn = 1.0 - 2.0 * (np.bitwise_count(j & zm) & 1)
        hp = (1j ** ny) * sgn * psi[j.astype(np.int64)]   # (P psi)[i]
        tot += float(np.real(cm * np.vdot(psi, hp)))
    return tot


def expm_evolve(H_dense: np.ndarray, psi: np.ndarray, t: float) -> np.ndarray:
    """exp(-iHt)|psi> in FP64 (dense; the reference's oracle, ab_test.py:435-441)."""
    import scipy.linalg
    return scipy.linalg.expm(-1j * H_dense * t) @ psi


def expm_multiply_evolve(H_sparse, psi: np.ndarray, t: float) -> np.ndarray:
    import scipy.sparse.linalg as spla
    return spla.expm_multiply(-1j * t * H_sparse, psi)


def energy(n: int, ops, params_row, x, z, c) -> float:
    """E(theta) in FP64 with the C oracle (rotation params substituted)."""
    ops = np.array(_ops(ops), copy=True)
    sel = ops["param"] >= 0
    ops["m"][sel, 0] = np.asarray(params_row, dtype=np.float64)[ops["param"][sel]]
    psi = simulate(n, ops)
    if n >= 14:
        return pauli_expectation_c(psi, x, z, c)
    return pauli_expectation(psi, x, z, c)


def grad_central_fd(n, ops, params_row, x, z, c, which, h=1e-3):
    out = []
    for p in which:
        tp = np.array(params_row, dtype=np.float64, copy=True)
        tm = tp.copy()
        tp[p] += h
        tm[p] -= h
        out.append((energy(n, ops, tp, x, z, c) - energy(n, ops, tm, x, z, c)) / (2 * h))
    return np.array(out)


def grad_param_shift(n, ops, params_row, x, z, c, which):
    out = []
    for p in which:
        tp = np.array(params_row, dtype=np.float64, copy=True)
        tm = tp.copy()
        tp[p] += math.pi / 2
        tm[p] -= math.pi / 2
        out.append(0.5 * (energy(n, ops, tp, x, z, c) - energy(n, ops, tm, x, z, c)))
    return np.array(out)


# ------------------------------------------------------------ noise channels
# Restatement of the reference's stochastic channels (bwk/csrc/noise_sm120.cu)
# for checking the trajectory runner.  Parity for this part is unpinned: the
# reference has no tests or fixtures for its noise kernels, so the checks
# rest on this restatement and on channel-level properties (trajectory
# averages against the Kraus-sum density matrix).
DEPOLARIZE, AMP_DAMP, DEPHASE = 20, 21, 22


def seed_uniforms(seed: int, count: int) -> np.ndarray:
    """splitmix64 from `seed`, top 53 bits -> [0, 1) (pure-Python loop)."""
    m = (1 << 64) - 1
    x, out = int(seed) & m, []
    for _ in range(int(count)):
        x = (x + 0x9E3779B97F4A7C15) & m
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
        z ^= z >> 31
        out.append((z >> 11) * 2.0 ** -53)
    return np.array(out, dtype=np.float64)


def depol_branch(p: float, u: float) -> int:
    """noise_sm120.cu:262-289: [0, 1-p) identity, then X, Y, Z in thirds of p."""
    if u < 1.0 - p:
        return 0
    r, third = u - (1.0 - p), p / 3.0
    if r < third:
        return 1
    if r < 2.0 * third:
        return 2
    return 3


def apply_channel_np(psi: np.ndarray, n: int, kind: int, q: int, g: float, u: float):
    """One channel on an FP64 state: (new state, branch, |u - p1|).
    Depolarizing: Pauli by depol_branch.  Damping / dephasing: jump when
    u < p1 = g P(q=1) (noise_sm120.cu:116-147, 296-312), Kraus operator of the
    branch, renormalised.  The damping jump is E1 = [[0, sqrt g], [0, 0]]."""
    psi = np.array(psi, dtype=np.complex128, copy=True)
    idx = np.arange(1 << n, dtype=np.int64)
    one = ((idx >> q) & 1) == 1
    if kind == DEPOLARIZE:
        b = depol_branch(g, u)
        P = [None, [[0, 1], [1, 0]], [[0, -1j], [1j, 0]], [[1, 0], [0, -1]]][b]
        if P is not None:
            psi = _apply_k(psi, n, [q], np.array(P, dtype=complex))
        return psi, b, math.inf
    S1 = float(np.sum(np.abs(psi[one]) ** 2))
    S0 = float(np.sum(np.abs(psi[~one]) ** 2))
    p1 = g * S1 / (S0 + S1)
    keep = S0 + (1.0 - g) * S1
    jump = S1 > 0.0 and (u < p1 or not keep > 0.0)
    if not jump:
        psi[~one] /= math.sqrt(keep)
        psi[one] *= math.sqrt(1.0 - g) / math.sqrt(keep)
    elif kind == AMP_DAMP:
        psi[~one] = psi[one] / math.sqrt(S1)
        psi[one] = 0
    else:
        psi[~one] = 0
        psi[one] /= math.sqrt(S1)
    return psi, int(jump), abs(u - p1)


def noise_trajectory(n: int, ops, seed: int):
    """One trajectory of a circuit with channel ops: (FP64 state, branches,
    smallest |u - p1| over the state-dependent channels)."""
    recs = _ops(ops)
    nn = int(sum(1 for r in recs if int(r["kind"]) in (DEPOLARIZE, AMP_DAMP, DEPHASE)))
    u = seed_uniforms(seed, nn)
    psi = zero_state(n)
    br, margin, k, pending = [], math.inf, 0, []
    for r in recs:
        kind = int(r["kind"])
        if kind in (DEPOLARIZE, AMP_DAMP, DEPHASE):
            if pending:
                psi = apply_ops_np(psi, n, np.array(pending, dtype=OP_DTYPE))
                pending = []
            psi, b, mg = apply_channel_np(psi, n, kind, int(r["q"][0]), float(r["m"][0]), float(u[k]))
            br.append(b)
            margin = min(margin, mg)
            k += 1
        else:
            pending.append(r)
    if pending:
        psi = apply_ops_np(psi, n, np.array(pending, dtype=OP_DTYPE))
    return psi, np.array(br, dtype=np.uint8), margin


def kraus_density(n: int, ops) -> np.ndarray:
    """Exact density matrix of the channel circuit (Kraus sums, FP64; n <= 6)."""
    recs = _ops(ops)
    N = 1 << n
    rho = np.zeros((N, N), dtype=np.complex128)
    rho[0, 0] = 1
    eye = np.eye(N, dtype=complex)
    for r in recs:
        kind, q = int(r["kind"]), int(r["q"][0])
        if kind in (DEPOLARIZE, AMP_DAMP, DEPHASE):
            g = float(r["m"][0])
            if kind == DEPOLARIZE:
                Ks = [math.sqrt(1 - g) * np.eye(2)] + [math.sqrt(g / 3) * np.array(P, dtype=complex) for P in
                                                       ([[0, 1], [1, 0]], [[0, -1j], [1j, 0]], [[1, 0], [0, -1]])]
            elif kind == AMP_DAMP:
                Ks = [np.array([[1, 0], [0, math.sqrt(1 - g)]]), np.array([[0, math.sqrt(g)], [0, 0]])]
            else:
                Ks = [np.array([[1, 0], [0, math.sqrt(1 - g)]]), np.array([[0, 0], [0, math.sqrt(g)]])]
            new = np.zeros_like(rho)
            for K in Ks:
                Kf = np.stack([_apply_k(eye[:, j].copy(), n, [q], np.asarray(K, dtype=complex)) for j in range(N)],
                              axis=1)
                new += Kf @ rho @ Kf.conj().T
            rho = new
        else:
            U = np.stack([apply_ops_np(eye[:, j], n, np.array([r], dtype=OP_DTYPE)) for j in range(N)], axis=1)
            rho = U @ rho @ U.conj().T
    return rho


def reference_amp_damp_jump(psi: np.ndarray, n: int, q: int, g: float) -> np.ndarray:
    """The reference's damping jump kernel as written (noise_sm120.cu:183-205,
    renorm 1/sqrt(p1) with p1 = g P(q=1), noise_sm120.cu:358-365): it keeps
    a0 * renorm in the |0> amplitudes, so the result is not E1|psi>/|E1 psi|."""
    psi = np.array(psi, dtype=np.complex128, copy=True)
    idx = np.arange(1 << n, dtype=np.int64)
    one = ((idx >> q) & 1) == 1
    p1 = g * float(np.sum(np.abs(psi[one]) ** 2))
    renorm = 1.0 / math.sqrt(p1)
    i1 = idx[one]
    i0 = i1 & ~(1 << q)
    psi[i0] = psi[i0] * renorm + psi[i1] * math.sqrt(g) * renorm
    psi[i1] = 0
    return psi
