"""Pin the FP64 oracle (and the host-side algorithm restatements) against the
reference's own outputs (tests/golden, made by tests/golden/make_golden.py)
and the reference's analytic checks (tests/stress_test.py)."""
import math
import os

import numpy as np
import pytest

import sv_oracle as O
from qsim_b200 import workloads as W
from qsim_b200.circuit import OP_DTYPE, Circuit, lower
from qsim_b200.paulis import PauliSum, csr_from_paulis

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _qv_ops_from(mats, qubits):
    G = qubits.shape[0]
    ops = np.zeros(G, dtype=OP_DTYPE)
    ops["kind"] = O.U2
    ops["nq"] = 2
    ops["param"] = -1
    ops["q"][:, :2] = qubits
    flat = mats.reshape(G, 16).astype(np.complex128)
    ops["m"][:, 0:32:2] = flat.real
    ops["m"][:, 1:32:2] = flat.imag
    return ops


def test_oracle_matches_reference_qv8():
    d = np.load(os.path.join(GOLD, "qv8_ref.npz"))
    gm, gq, probs = d["gate_matrices"], d["gate_qubits"], d["probs"]
    for c in range(gm.shape[0]):
        mats = gm[c, ..., 0] + 1j * gm[c, ..., 1]
        psi = O.simulate(8, _qv_ops_from(mats, gq[c]))
        # reference probabilities are FP32 (torch complex64)
        np.testing.assert_allclose(np.abs(psi) ** 2, probs[c], atol=2e-6)


def test_oracle_matches_reference_qv4():
    d = np.load(os.path.join(GOLD, "qv4_ref.npz"))
    pairs = np.array([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)])
    for c in range(d["gate_data"].shape[0]):
        gd = d["gate_data"][c]
        mats = (gd[:, :16] + 1j * gd[:, 16:]).reshape(-1, 4, 4)
        psi = O.simulate(4, _qv_ops_from(mats, pairs[d["pair_ids"][c]]))
        np.testing.assert_allclose(np.abs(psi) ** 2, d["probs"][c], atol=2e-6)


def test_chebyshev_coefficients_match_reference():
    from blackwell_backend.chebyshev import chebyshev_coefficients
    d = np.load(os.path.join(GOLD, "cheb_coeffs_ref.npz"))
    for i in range(int(d["n"])):
        t, b, p, K, tail = d[f"meta{i}"]
        c, K2, tail2 = chebyshev_coefficients(t, b, p)
        assert K2 == int(K)
        assert tail2 == tail
        np.testing.assert_array_equal(c, d[f"c{i}"])


def _random_ops(n, count, rng):
    """Random mix of every op kind."""
    recs = np.zeros(count, dtype=OP_DTYPE)
    for k in range(count):
        r = recs[k]
        r["param"] = -1
        kind = int(rng.integers(1, 14))
        need = {O.U1: 1, O.U2: 2, O.DIAG1: 1, O.DIAG2: 2, O.MCU1: 2, O.MCU2: 3, O.MCX: 3, O.MCSWAP: 3,
                O.MCPHASE: 2, O.Y: 1, O.RX: 1, O.RY: 1, O.RZ: 1}[kind]
        nq = min(n, need + (int(rng.integers(0, 2)) if kind in (O.MCU1, O.MCX, O.MCPHASE) else 0))
        if nq < need:
            kind, nq = O.U1, 1
        q = rng.choice(n, nq, replace=False)
        r["kind"], r["nq"] = kind, nq
        r["q"][:nq] = q
        if kind in (O.U1, O.MCU1):
            m = W.G.haar_unitary(rng, 2)
        elif kind in (O.U2, O.MCU2):
            m = W.G.haar_unitary(rng, 4)
        elif kind == O.DIAG1:
            m = np.exp(1j * rng.uniform(0, 6.3, 2))
        elif kind == O.DIAG2:
            m = np.exp(1j * rng.uniform(0, 6.3, 4))
        elif kind == O.MCPHASE:
            m = np.exp(1j * rng.uniform(0, 6.3, 1))
        elif kind in (O.RX, O.RY, O.RZ):
            r["m"][0] = rng.uniform(-4, 4)
            continue
        else:
            continue
        flat = np.asarray(m).reshape(-1)
        r["m"][: 2 * flat.size: 2] = flat.real
        r["m"][1: 2 * flat.size: 2] = flat.imag
    return recs


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8])
def test_c_oracle_equals_numpy_oracle(n):
    rng = np.random.default_rng(100 + n)
    ops = _random_ops(n, 60, rng)
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi0 /= np.linalg.norm(psi0)
    a = O.simulate(n, ops, psi0)
    b = O.apply_ops_np(psi0, n, ops)
    np.testing.assert_allclose(a, b, atol=1e-12)


def test_lowering_matches_dense_matrices():
    """Circuit -> ops -> oracle equals an independent Kronecker-product build."""
    from qsim_b200 import gates as G
    n = 3
    qc = Circuit(n)
    qc.h(0).rx(0.3, 1).cx(0, 2).cz(1, 2).swap(0, 1).cp(0.7, 2, 0).crz(1.1, 0, 1).u(0.2, 0.4, 0.6, 2).ccx(0, 1, 2)
    qc.cu(0.3, 0.2, 0.1, 0.5, 2, 1).cswap(2, 0, 1).t(1).sdg(0).sx(2).y(1).unitary(G.haar_unitary(
        np.random.default_rng(3), 4), [2, 0])
    psi = O.simulate(n, lower(qc))

    def embed(name, qs, params=(), mat=None):
        # dense 2^n operator with matrix index bit j = qs[j]
        if mat is None:
            if len(qs) == 1:
                mat = G.mat1(name, params)
            elif name in G.NATIVE_2Q:
                mat = G.mat2_little(name, params)
            elif name == "ccx":
                mat = np.eye(8, dtype=complex)
                mat[[3, 7]] = mat[[7, 3]]
            elif name == "cswap":
                mat = np.eye(8, dtype=complex)
                mat[[3, 5]] = mat[[5, 3]]
        k = len(qs)
        N = 1 << n
        U = np.zeros((N, N), dtype=complex)
        for col in range(N):
            sub = sum(((col >> q) & 1) << j for j, q in enumerate(qs))
            for r in range(1 << k):
                row = col
                for j, q in enumerate(qs):
                    row = (row & ~(1 << q)) | (((r >> j) & 1) << q)
                U[row, col] += mat[r, sub]
        return U

    ref = np.zeros(1 << n, dtype=complex)
    ref[0] = 1
    for ins in qc.data:
        ref = embed(ins.name, ins.qubits, ins.params, ins.matrix) @ ref
    np.testing.assert_allclose(psi, ref, atol=1e-12)


def test_analytic_pins_on_oracle():
    """GHZ, H^1000 = I, X^999 = X, CX^1000 (tests/stress_test.py:463-817)."""
    n = 6
    qc = Circuit(n)
    qc.h(0)
    for q in range(n - 1):
        qc.cx(q, q + 1)
    psi = O.simulate(n, lower(qc))
    assert abs(abs(psi[0]) ** 2 - 0.5) < 1e-12 and abs(abs(psi[-1]) ** 2 - 0.5) < 1e-12
    qc = Circuit(4)
    for _ in range(1000):
        qc.h(2)
    assert abs(O.simulate(4, lower(qc))[0] - 1) < 1e-9
    qc = Circuit(4)
    for _ in range(999):
        qc.x(1)
    assert abs(O.simulate(4, lower(qc))[2] - 1) < 1e-12


def test_workload_shapes():
    assert len(W.qv_ops(12, 12, 0)) == 72
    ops = W.layers_ops(32, 20, 0)
    kinds = np.bincount(ops["kind"], minlength=14)
    assert kinds[O.U1] == 640 and kinds[O.MCPHASE] == 310 and kinds[O.MCX] == 4 and len(ops) == 954
    w, oo, ops2, so = W.qv_batch(64, 10, 20, 5)
    assert w.min() >= 10 and w.max() <= 20 and oo[-1] == len(ops2)
    assert np.all(np.diff(so) == (1 << w[:-1].astype(np.int64)))
    qc, npar = W.efficient_su2(20, 4)
    assert npar == 200 and qc.size() == 200 + 4 * 19


def test_csr_builder_matches_dense():
    ps = W.serving_hamiltonian(6, seed=3, n_pairs=5)
    rp, ci, val = csr_from_paulis(ps)
    import scipy.sparse as sp
    A = sp.csr_matrix((val.astype(np.complex128), ci, rp), shape=(64, 64)).toarray()
    np.testing.assert_allclose(A, ps.to_dense(), atol=1e-7)
    # Heisenberg chain from labels (ab_test.py:382-393)
    terms = []
    for i in range(4):
        for p in "XYZ":
            lab = ["I"] * 5
            lab[i] = lab[i + 1] = p
            terms.append(("".join(lab), 0.5))
    h = PauliSum.from_list(terms)
    rp, ci, val = csr_from_paulis(h)
    A = sp.csr_matrix((val.astype(np.complex128), ci, rp), shape=(32, 32)).toarray()
    np.testing.assert_allclose(A, h.to_dense(), atol=1e-7)
    np.testing.assert_allclose(A, A.conj().T, atol=1e-7)


def test_oracle_sampling_and_expectation_semantics():
    rng = np.random.default_rng(0)
    psi = rng.standard_normal(16) + 1j * rng.standard_normal(16)
    psi /= np.linalg.norm(psi)
    cdf = np.cumsum(np.abs(psi) ** 2)
    u = np.array([0.0, cdf[3], cdf[3] + 1e-9, 0.999999999, 2.0])
    s = O.sample_indices(psi, u)
    assert list(s) == [0, 3, 4, int(np.searchsorted(cdf, 0.999999999)), 15]
    # <Z0> = P(0) - P(1); <X0> = 2 Re(sum conj(a0) a1)
    z = O.pauli_expectation(psi, [0], [1], [1.0])
    p = np.abs(psi) ** 2
    assert abs(z - (p[0::2].sum() - p[1::2].sum())) < 1e-12
    x = O.pauli_expectation(psi, [1], [0], [1.0])
    assert abs(x - 2 * np.real(np.vdot(psi[0::2], psi[1::2]))) < 1e-12
    y = O.pauli_expectation(psi, [1], [1], [1.0])
    Y = np.kron(np.eye(8), np.array([[0, -1j], [1j, 0]]))
    assert abs(y - np.real(np.vdot(psi, Y @ psi))) < 1e-12


@pytest.mark.parametrize("n", [3, 9, 14])
def test_c_pauli_expectation_equals_numpy(n):
    """The C oracle's Pauli-sum expectation (used for 20+ qubits) against the
    numpy restatement, X/Y/Z strings of weight 1-4 with Y phases."""
    rng = np.random.default_rng(n)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    ps = W.random_pauli_observable(n, 48, seed=n + 1, wmax=min(4, n))
    a = O.pauli_expectation(psi, ps.x, ps.z, ps.real_coefs())
    b = O.pauli_expectation_c(psi, ps.x, ps.z, ps.real_coefs())
    assert abs(a - b) <= 1e-12 * max(1.0, abs(a))
