"""CPU checks of the noise-channel restatement in the oracle: its uniforms
match the library's seeded stream, its trajectory average converges to the
Kraus-sum density matrix, and the reference's damping jump kernel (as
written) does not give a normalised E1 state — the reason the library's jump
branch differs from it."""
import math

import numpy as np

import sv_oracle as O
from qsim_b200.circuit import Circuit, lower
from qsim_b200.engine import seed_uniforms
from qsim_b200.noise import add_noise


def _circ():
    qc = Circuit(3)
    qc.h(0)
    qc.cx(0, 1)
    qc.ry(0.7, 2)
    qc.cx(1, 2)
    return add_noise(qc, depolarizing=0.08, amplitude_damping=0.15, dephasing=0.1)


def test_uniform_streams_agree():
    for s in (0, 5, 2 ** 63 + 11):
        assert np.array_equal(O.seed_uniforms(s, 50), seed_uniforms(s, 50))


def test_depol_branch_ranges():
    p = 0.3
    assert O.depol_branch(p, 0.0) == 0 and O.depol_branch(p, 0.6999) == 0
    assert O.depol_branch(p, 0.7) == 1 and O.depol_branch(p, 0.79) == 1
    assert O.depol_branch(p, 0.81) == 2 and O.depol_branch(p, 0.91) == 3
    assert O.depol_branch(0.0, 0.999999) == 0


def test_channel_edge_cases():
    one = np.zeros(2, dtype=complex)
    one[1] = 1
    psi, b, _ = O.apply_channel_np(one, 1, O.AMP_DAMP, 0, 1.0, 0.5)
    assert b == 1 and np.allclose(psi, [1, 0])               # full decay
    zero = np.array([1, 0], dtype=complex)
    psi, b, _ = O.apply_channel_np(zero, 1, O.AMP_DAMP, 0, 0.7, 0.0)
    assert b == 0 and np.allclose(psi, [1, 0])               # nothing to decay
    plus = np.array([1, 1], dtype=complex) / math.sqrt(2)
    psi, b, _ = O.apply_channel_np(plus, 1, O.DEPHASE, 0, 0.5, 0.99)
    assert b == 0 and abs(np.linalg.norm(psi) - 1) < 1e-15


def test_trajectory_average_matches_kraus_density():
    qc = _circ()
    ops = lower(qc)
    rho = O.kraus_density(3, ops)
    assert abs(np.trace(rho) - 1) < 1e-12
    T = 3000
    acc = np.zeros_like(rho)
    for t in range(T):
        psi, _, _ = O.noise_trajectory(3, ops, 1000 + t)
        assert abs(np.linalg.norm(psi) - 1) < 1e-12
        acc += np.outer(psi, psi.conj())
    acc /= T
    # each entry is a mean of T terms bounded by 1: 5 sigma ~ 5 / sqrt(T)
    assert np.max(np.abs(acc - rho)) < 5 / math.sqrt(T)


def test_reference_damping_jump_is_not_normalised():
    plus = np.array([1, 1], dtype=complex) / math.sqrt(2)
    ref = O.reference_amp_damp_jump(plus, 1, 0, 0.3)
    ours, b, _ = O.apply_channel_np(plus, 1, O.AMP_DAMP, 0, 0.3, 0.0)
    assert b == 1 and np.allclose(ours, [1, 0])
    assert abs(np.linalg.norm(ref) - 1) > 0.5


def test_add_noise_inserts_channels():
    from qsim_b200.noise import n_channels
    qc = Circuit(3)
    qc.h(0)
    qc.cx(0, 1)
    qc.barrier()
    qc.measure(1, 0) if qc.num_clbits else None
    noisy = add_noise(qc, depolarizing=0.01, amplitude_damping=0.02)
    assert [i.name for i in noisy.data] == ["h", "depolarize", "amplitude_damp", "cx", "depolarize",
                                            "amplitude_damp", "depolarize", "amplitude_damp", "barrier"]
    assert n_channels(noisy) == 6
    assert list(lower(noisy)["kind"]) == [1, 20, 21, 7, 20, 21, 20, 21]
