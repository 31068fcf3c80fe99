"""The planner's device program, emulated on the host in FP64 (no GPU),
against the FP64 oracle: fusion, rotation decomposition into scaled
rotations + merged diagonal tables, Kronecker layers, controls on register
and global qubits and the pass split must reproduce the circuit to the
precision of the FP32 coefficients."""
import numpy as np
import pytest

import __graft_entry__  # noqa: F401
import plan_emulator as PE
import sv_oracle as O
from qsim_b200 import workloads as W
from test_oracle_golden import _random_ops


def _check(n, ops, tile_bits, block_bits, psi0=None, specialised=False):
    blob = PE.program(n, ops, tile_bits, block_bits, specialised)
    if psi0 is None:
        psi0 = np.zeros(1 << n, complex)
        psi0[0] = 1
    got = PE.run(n, blob, psi0)
    ref = O.simulate(n, ops, psi0)
    assert abs(1 - O.fidelity(got, ref)) <= 1e-12
    assert np.abs(got - ref).max() <= 1e-6
    return len(PE.decode(blob))


@pytest.mark.parametrize("specialised", [False, True])
@pytest.mark.parametrize("n,tile_bits,block_bits", [(3, 10, 5), (6, 10, 5), (10, 10, 4), (12, 10, 3),
                                                    (13, 10, 5), (12, 10, 2), (13, 11, 5)])
def test_random_all_kinds(n, tile_bits, block_bits, specialised):
    rng = np.random.default_rng(7000 + n)
    ops = _random_ops(n, 100, rng)
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    _check(n, ops, tile_bits, block_bits, psi0 / np.linalg.norm(psi0), specialised)


@pytest.mark.parametrize("tile_bits,block_bits", [(10, 5), (12, 4), (11, 3)])
def test_layered_brickwork_multipass(tile_bits, block_bits):
    assert _check(16, W.layers_ops(16, 8, seed=3), tile_bits, block_bits) > 1


@pytest.mark.parametrize("specialised", [False, True])
def test_qv(specialised):
    _check(12, W.qv_ops(12, 12, 0), 10, 5, specialised=specialised)


def test_scale_folding_long_rotation_chain():
    """Hundreds of scaled rotations in one pass: the dropped factors must be
    folded back (tables / explicit scale ops) without leaving FP32 range."""
    n = 10
    rng = np.random.default_rng(11)
    recs = np.zeros(600, dtype=W.OP_DTYPE)
    for k in range(600):
        r = recs[k]
        r["kind"], r["nq"], r["param"] = 12, 1, -1   # QS_OP_RY
        r["q"][0] = k % n
        r["m"][0] = rng.uniform(0.3, 2.8)
    _check(n, recs, 10, 5)


def _u2_record(m, q0, q1):
    from qsim_b200.circuit import OP_DTYPE
    r = np.zeros(1, dtype=OP_DTYPE)
    r["kind"], r["nq"], r["param"] = 2, 2, -1
    r["q"][0, 0], r["q"][0, 1] = q0, q1
    flat = np.asarray(m, dtype=np.complex128).reshape(-1)
    r["m"][0, :32:2] = flat.real
    r["m"][0, 1:32:2] = flat.imag
    return r


def test_cartan_split_special_two_qubit_gates():
    """Dense 4x4 gates with degenerate Cartan forms (product, diagonal, CNOT,
    SWAP, iSWAP, sqrt(SWAP), identity) and random ones, on both qubit orders."""
    rng = np.random.default_rng(21)
    I2 = np.eye(2)
    X = np.array([[0, 1], [1, 0]])
    H = np.array([[1, 1], [1, -1]]) / np.sqrt(2)
    cnot = np.array([[1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0], [0, 1, 0, 0]])
    swap = np.eye(4)[[0, 2, 1, 3]]
    iswap = np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]])
    sq = np.array([[1, 0, 0, 0], [0, (1 + 1j) / 2, (1 - 1j) / 2, 0], [0, (1 - 1j) / 2, (1 + 1j) / 2, 0], [0, 0, 0, 1]])
    mats = [np.eye(4), np.kron(H, X), np.diag(np.exp(1j * rng.uniform(0, 6, 4))), cnot, swap, iswap, sq,
            np.kron(I2, H) @ cnot]
    mats += [W.G.haar_unitary(rng, 4) for _ in range(6)]
    n = 6
    recs = []
    for k, m in enumerate(mats):
        q0, q1 = (k % n, (k * 3 + 1) % n) if k % 2 else ((k * 3 + 1) % n, k % n)
        if q0 == q1:
            q1 = (q0 + 1) % n
        recs.append(_u2_record(m, q0, q1))
        recs.append(_u2_record(W.G.haar_unitary(rng, 4), (q0 + 2) % n, (q1 + 3) % n)
                    if (q0 + 2) % n != (q1 + 3) % n else _u2_record(np.eye(4), 0, 1))
    ops = np.concatenate(recs)
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    _check(n, ops, 10, 5, psi0 / np.linalg.norm(psi0), specialised=True)


@pytest.mark.parametrize("n,tile_bits", [(14, 10), (16, 12)])
def test_six_qubit_register_blocks(n, tile_bits):
    """Specialised plans may use 6-qubit register blocks (64-bit register
    masks in the diagonal tables)."""
    rng = np.random.default_rng(9100 + n)
    ops = np.concatenate([W.layers_ops(n, 6, seed=5), _random_ops(n, 60, rng)])
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    _check(n, ops, tile_bits, 6, psi0 / np.linalg.norm(psi0), specialised=True)


def test_dense_only_passes_are_marked():
    """Passes whose device ops are all uncontrolled dense 4x4s carry has2 = 2
    (the interpreter's dispatch-free op loop); any other op kind keeps 1 or 0,
    and the program still matches the oracle."""
    ops = W.qv_ops(16, 16, 3)
    blob = PE.program(16, ops, 13, 4, False)
    dec = PE.decode(blob)
    assert all(int(h["has2"]) == 2 for h, _, dops, _ in dec)
    assert all(int(o["kind"]) == PE.DK_U2 for _, _, dops, _ in dec for o in dops)
    _check(16, ops, 13, 4)
    lay = W.layers_ops(16, 4, seed=1)
    for h, _, dops, _ in PE.decode(PE.program(16, lay, 13, 4, False)):
        assert int(h["has2"]) in (0, 1)
