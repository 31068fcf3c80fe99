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


def _check(n, ops, tile_bits, block_bits, psi0=None):
    blob = PE.program(n, ops, tile_bits, block_bits)
    if psi0 is None:
        psi0 = np.zeros(1 << n, complex)
        psi0[0] = 1
    got = PE.run(n, blob, psi0)
    ref = O.simulate(n, ops, psi0)
    assert abs(1 - O.fidelity(got, ref)) <= 1e-12
    assert np.abs(got - ref).max() <= 1e-6
    return len(PE.decode(blob))


@pytest.mark.parametrize("n,tile_bits,block_bits", [(3, 10, 5), (6, 10, 5), (10, 10, 4), (12, 10, 3),
                                                    (13, 10, 5), (12, 10, 2), (13, 11, 5)])
def test_random_all_kinds(n, tile_bits, block_bits):
    rng = np.random.default_rng(7000 + n)
    ops = _random_ops(n, 100, rng)
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    _check(n, ops, tile_bits, block_bits, psi0 / np.linalg.norm(psi0))


@pytest.mark.parametrize("tile_bits,block_bits", [(10, 5), (12, 4), (11, 3)])
def test_layered_brickwork_multipass(tile_bits, block_bits):
    assert _check(16, W.layers_ops(16, 8, seed=3), tile_bits, block_bits) > 1


def test_qv():
    _check(12, W.qv_ops(12, 12, 0), 10, 5)


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
