"""GPU parity of the one-gate-per-launch kernels (the reference's per-op API)
against the FP64 oracle; exact permutation kernels bit for bit."""
import itertools

import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200.circuit import OP_DTYPE

pytestmark = pytest.mark.gpu

TOL = 2e-6  # max |amp error| for one compensated gate on a normalised state


def rand_state(n, seed):
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return (psi / np.linalg.norm(psi)).astype(np.complex64)


def dev(psi):
    return torch.from_numpy(psi.copy()).cuda()


def op(kind, qs, m=None):
    r = np.zeros(1, dtype=OP_DTYPE)
    r["kind"], r["nq"], r["param"] = kind, len(qs), -1
    r["q"][0, : len(qs)] = qs
    if m is not None:
        f = np.asarray(m, dtype=np.complex128).reshape(-1)
        r["m"][0, : 2 * f.size: 2] = f.real
        r["m"][0, 1: 2 * f.size: 2] = f.imag
    return r


def haar(d, seed):
    from qsim_b200.gates import haar_unitary
    return haar_unitary(np.random.default_rng(seed), d)


@pytest.mark.parametrize("n", [1, 2, 5, 10, 13])
def test_apply_gate_all_targets(n):
    import blackwell_kernels as bk
    for t in range(n):
        psi = rand_state(n, t)
        U = haar(2, 100 + t)
        s = dev(psi)
        bk.apply_gate(s, torch.from_numpy(U.astype(np.complex64)), t)
        ref = O.simulate(n, op(O.U1, [t], U.astype(np.complex64).astype(np.complex128)), psi.astype(np.complex128))
        assert np.max(np.abs(s.cpu().numpy() - ref)) < TOL


@pytest.mark.parametrize("n", [2, 3, 8, 12])
def test_apply_gate_2q_all_pairs(n):
    import blackwell_kernels as bk
    for a, b in itertools.permutations(range(n), 2):
        if n > 8 and (a + b) % 3:
            continue
        psi = rand_state(n, 7 * a + b)
        U = haar(4, a * 31 + b).astype(np.complex64)
        s = dev(psi)
        bk.apply_gate_2q(s, torch.from_numpy(U), a, b)
        # reference semantics: bit 0 of the 4x4 index is min(a, b)
        ref = O.simulate(n, op(O.U2, [min(a, b), max(a, b)], U.astype(np.complex128)), psi.astype(np.complex128))
        assert np.max(np.abs(s.cpu().numpy() - ref)) < TOL, (a, b)


@pytest.mark.parametrize("n", [3, 9])
def test_diagonals_and_phase(n):
    import blackwell_kernels as bk
    rng = np.random.default_rng(5)
    for t in range(n):
        psi = rand_state(n, t)
        d = np.exp(1j * rng.uniform(0, 6.28, 2)).astype(np.complex64)
        s = dev(psi)
        bk.apply_diagonal(s, torch.from_numpy(d), t)
        ref = O.simulate(n, op(O.DIAG1, [t], d.astype(np.complex128)), psi.astype(np.complex128))
        assert np.max(np.abs(s.cpu().numpy() - ref)) < TOL
        ph = complex(np.exp(1j * rng.uniform(0, 6.28)).astype(np.complex64))
        s = dev(psi)
        bk.apply_diagonal_phase(s, ph, t)
        ref = O.simulate(n, op(O.MCPHASE, [t], [ph]), psi.astype(np.complex128))
        assert np.max(np.abs(s.cpu().numpy() - ref)) < TOL
    for a, b in [(0, 1), (1, n - 1), (n - 1, 0)]:
        psi = rand_state(n, a + 10 * b)
        d = np.exp(1j * rng.uniform(0, 6.28, 4)).astype(np.complex64)
        s = dev(psi)
        bk.apply_diagonal_2q(s, torch.from_numpy(d), a, b)
        ref = O.simulate(n, op(O.DIAG2, [min(a, b), max(a, b)], d.astype(np.complex128)), psi.astype(np.complex128))
        assert np.max(np.abs(s.cpu().numpy() - ref)) < TOL


def test_multicontrolled_dense():
    import blackwell_kernels as bk
    n = 7
    for k, (ctrl, t) in enumerate([([0], 3), ([2, 5], 0), ([6, 1, 3], 4), ([0, 1, 2, 3, 4, 5], 6)]):
        psi = rand_state(n, k)
        U = haar(2, 50 + k).astype(np.complex64)
        s = dev(psi)
        bk.apply_mcgate(s, torch.from_numpy(U), ctrl, t)
        ref = O.simulate(n, op(O.MCU1, ctrl + [t], U.astype(np.complex128)), psi.astype(np.complex128))
        assert np.max(np.abs(s.cpu().numpy() - ref)) < TOL
    for k, (ctrl, a, b) in enumerate([([0], 3, 5), ([6, 2], 1, 0)]):
        psi = rand_state(n, 20 + k)
        U = haar(4, 70 + k).astype(np.complex64)
        s = dev(psi)
        bk.apply_mc2qgate(s, torch.from_numpy(U), ctrl, a, b)
        ref = O.simulate(n, op(O.MCU2, ctrl + [min(a, b), max(a, b)], U.astype(np.complex128)),
                         psi.astype(np.complex128))
        assert np.max(np.abs(s.cpu().numpy() - ref)) < TOL


def _perm_ref(psi, n, f):
    """out[f(i)] = psi[i] for a basis permutation f (numpy, exact)."""
    out = np.empty_like(psi)
    idx = np.arange(1 << n)
    out[f(idx)] = psi
    return out


def _eq_bits(a, b):
    # +0 and -0 are treated as equal
    return np.array_equal(a.view(np.float32) + 0.0, b.view(np.float32) + 0.0)


def test_exact_permutations_bit_exact():
    """X, CNOT (all 56 ordered pairs on 8 qubits), SWAP, Toffoli (all triples on
    6 qubits), CZ: values moved or negated bit-exactly (the reference's 0/1
    dense kernels reproduce moved values exactly, stress_test.py:217-257,583-603)."""
    import blackwell_kernels as bk
    n = 8
    psi = rand_state(n, 1)
    for t in range(n):
        s = dev(psi)
        bk.apply_mcgate(s, bk.pauli_x_gate(), [], t)
        assert _eq_bits(s.cpu().numpy(), _perm_ref(psi, n, lambda i: i ^ (1 << t)))
    for c, t in itertools.permutations(range(n), 2):
        s = dev(psi)
        bk.apply_mcgate(s, bk.pauli_x_gate(), [c], t)
        assert _eq_bits(s.cpu().numpy(), _perm_ref(psi, n, lambda i: i ^ (((i >> c) & 1) << t)))
    for a, b in itertools.combinations(range(n), 2):
        s = dev(psi)
        bk.apply_mc2qgate(s, bk.swap_gate(), [], a, b)
        sw = lambda i: i ^ ((((i >> a) ^ (i >> b)) & 1) * ((1 << a) | (1 << b)))
        assert _eq_bits(s.cpu().numpy(), _perm_ref(psi, n, sw))
        s = dev(psi)
        bk.apply_gate_2q(s, bk.cz_gate(), a, b)
        ref = psi.copy()
        idx = np.arange(1 << n)
        ref[((idx >> a) & 1) & ((idx >> b) & 1) == 1] *= -1
        assert _eq_bits(s.cpu().numpy(), ref)
    m = 6
    psi6 = rand_state(m, 2)
    for c1, c2, t in itertools.permutations(range(m), 3):
        s = dev(psi6)
        bk.apply_mcgate(s, bk.pauli_x_gate(), [c1, c2], t)
        f = lambda i: i ^ ((((i >> c1) & (i >> c2)) & 1) << t)
        assert _eq_bits(s.cpu().numpy(), _perm_ref(psi6, m, f))


def test_state_init_and_batched():
    import blackwell_kernels as bk
    s = bk.state_init(11).cpu().numpy()
    assert s[0] == 1 and np.count_nonzero(s) == 1
    B = bk.state_init_batched(5, 6)
    assert B.shape == (5, 64)
    U = haar(2, 9).astype(np.complex64)
    bk.apply_gate_batched(B, torch.from_numpy(U), 4)
    ref = O.simulate(6, op(O.U1, [4], U.astype(np.complex128)))
    for b in range(5):
        assert np.max(np.abs(B[b].cpu().numpy() - ref)) < TOL
    gates = np.stack([haar(2, k) for k in range(6)]).astype(np.complex64)
    tg = torch.tensor([0, 1, 2, 3, 4, 5], dtype=torch.int32)
    B2 = bk.state_init_batched(3, 6)
    bk.apply_gates_batched_fused(B2, torch.from_numpy(gates), tg)
    ops = np.concatenate([op(O.U1, [k], gates[k].astype(np.complex128)) for k in range(6)])
    ref = O.simulate(6, ops)
    for b in range(3):
        assert np.max(np.abs(B2[b].cpu().numpy() - ref)) < 1e-5


def test_errors_are_raised_not_silent():
    import blackwell_kernels as bk
    s = bk.state_init(4)
    with pytest.raises(RuntimeError):
        bk.apply_gate(s, bk.hadamard_gate(), 7)
    with pytest.raises(RuntimeError):
        bk.apply_gate_2q(s, bk.cnot_gate(), 1, 1)
    with pytest.raises(RuntimeError):
        bk.apply_mcgate(s, bk.pauli_x_gate(), [2], 2)
