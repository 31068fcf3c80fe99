"""The whole-state noise-trajectory program, emulated on the host in FP64 (no
GPU), against the oracle's channel-by-channel trajectories: the grouping of
channels into noise blocks, the composed branch maps (histogram, in-order
decisions, one application) and the gate passes between them must give the
oracle's branches and state for the same seed."""
import numpy as np
import pytest

import __graft_entry__  # noqa: F401
import plan_emulator as PE
import sv_oracle as O
from qsim_b200 import workloads as W
from qsim_b200.circuit import Circuit, lower
from qsim_b200.noise import add_noise


def _check(n, ops, seeds, block_bits=0):
    blob = PE.noise_program(n, ops, block_bits)
    nblocks = sum(int(b["pos"][6]) for _, blocks, _, _ in PE.decode(blob) for b in blocks)
    compared = 0
    for seed in seeds:
        psi0 = np.zeros(1 << n, complex)
        psi0[0] = 1
        br = []
        got = PE.run(n, blob, psi0, seed=seed, branches=br)
        ref, ref_br, margin = O.noise_trajectory(n, ops, seed)
        got_br = np.zeros(len(ref_br), np.uint8)
        for k, b in br:
            got_br[k] = b
        assert sorted(k for k, _ in br) == list(range(len(ref_br)))   # every channel decided once
        if margin < 1e-6:        # a state-dependent draw too close to its threshold to compare
            continue
        compared += 1
        assert np.array_equal(got_br, ref_br)
        assert np.abs(got - ref).max() <= 2e-5
    return nblocks, compared


@pytest.mark.parametrize("n,layers", [(4, 4), (7, 3), (10, 2), (14, 1)])
def test_noisy_brickwork(n, layers):
    qc = W.noisy_brickwork(n, layers, seed=n, depolarizing=0.05, amplitude_damping=0.1, dephasing=0.1)
    nblocks, compared = _check(n, lower(qc), range(12))
    assert nblocks > 0 and compared >= 8


@pytest.mark.parametrize("block_bits", [0, 2, 3, 5])
def test_block_widths(block_bits):
    qc = W.noisy_brickwork(6, 3, seed=4, depolarizing=0.1, amplitude_damping=0.2, dephasing=0.15)
    _, compared = _check(6, lower(qc), range(8), block_bits)
    assert compared >= 5


def test_channel_only_circuit_and_certain_jumps():
    """No gates at all; then damping with g = 1 from |1>, a jump with
    probability 1, and depolarizing with p = 1 (never the identity)."""
    qc = Circuit(3)
    qc.depolarize(0.5, 0)
    qc.dephase(0.5, 2)
    _check(3, lower(qc), range(6))
    qc = Circuit(3)
    qc.x(1)
    qc.amplitude_damp(1.0, 1)
    qc.depolarize(1.0, 2)
    blob = PE.noise_program(3, lower(qc))
    for seed in range(6):
        br = []
        psi0 = np.zeros(8, complex)
        psi0[0] = 1
        got = PE.run(3, blob, psi0, seed=seed, branches=br)
        d = dict(br)
        assert d[0] == 1 and d[1] != 0
        assert abs(np.linalg.norm(got) - 1) < 1e-6
        assert np.abs(got[np.abs(got) > 1e-9].size) == 1


def test_many_channels_on_one_qubit_share_blocks():
    """More channels on one qubit than a block takes (32 ops): the program
    splits them over several blocks and the result still matches."""
    qc = Circuit(5)
    qc.h(0)
    for _ in range(40):
        qc.amplitude_damp(0.02, 0)
        qc.depolarize(0.01, 0)
    qc = add_noise(qc, dephasing=0.05)
    nblocks, compared = _check(5, lower(qc), range(6))
    assert nblocks >= 3 and compared >= 4


def test_rejects_wide_states():
    with pytest.raises(Exception):
        PE.noise_program(15, lower(W.noisy_brickwork(15, 1, seed=1)))
