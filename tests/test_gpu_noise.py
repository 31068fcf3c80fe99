"""Noise channels on the GPU against the oracle's FP64 restatement:
single-state channels (the reference's apply_depolarizing /
apply_amplitude_damping / apply_dephasing) and batched trajectories on both
paths (whole-state tiles up to 14 qubits; segment launches above), branch by
branch, with trajectories bit-identical alone and in a batch, and the
trajectory average converging to the Kraus-sum density matrix."""
import math

import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200.circuit import Circuit, lower
from qsim_b200.noise import add_noise, run_trajectories

pytestmark = pytest.mark.gpu

FID_TOL = 1e-6      # |1 - F| per trajectory against FP64
MARGIN = 1e-5       # |u - p1| below this the FP32 state may take the other branch


def _rand_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return (v / np.linalg.norm(v)).astype(np.complex64)


def _circuit(n, depth, seed, dep=0.05, amp=0.08, deph=0.06):
    rng = np.random.default_rng(seed)
    qc = Circuit(n, name=f"noisy{n}")
    for d in range(depth):
        for q in range(n):
            qc.ry(float(rng.uniform(0, 3)), q)
            qc.rz(float(rng.uniform(0, 3)), q)
        for q in range(d % 2, n - 1, 2):
            qc.cx(q, q + 1)
    return add_noise(qc, depolarizing=dep, amplitude_damping=amp, dephasing=deph)


@pytest.mark.parametrize("kind", ["amp", "deph"])
def test_single_state_channels_match_oracle(kind):
    import blackwell_kernels as bk
    n, q = 7, 3
    fn = bk.apply_amplitude_damping if kind == "amp" else bk.apply_dephasing
    okind = O.AMP_DAMP if kind == "amp" else O.DEPHASE
    for g in (0.0, 0.3, 1.0):
        for u in (0.01, 0.2, 0.6, 0.97):
            psi = _rand_state(n, 11)
            ref, b_ref, margin = O.apply_channel_np(psi.astype(np.complex128), n, okind, q, g, u)
            st = torch.from_numpy(psi).cuda()
            b = fn(st, q, g, u)
            if margin < MARGIN:
                continue
            assert b == b_ref, (g, u)
            out = st.cpu().numpy()
            assert np.max(np.abs(out - ref)) < 1e-6
            assert abs(np.linalg.norm(out.astype(np.complex128)) - 1) < 1e-6


def test_depolarizing_paulis_exact():
    import blackwell_kernels as bk
    n, q, p = 6, 4, 0.3
    psi = _rand_state(n, 5)
    for u, want in ((0.1, 0), (0.75, 1), (0.85, 2), (0.95, 3)):
        ref, b_ref, _ = O.apply_channel_np(psi.astype(np.complex128), n, O.DEPOLARIZE, q, p, u)
        st = torch.from_numpy(psi).cuda()
        assert bk.apply_depolarizing(st, q, p, u) == b_ref == want
        assert np.array_equal(st.cpu().numpy(), ref.astype(np.complex64))   # exact: swaps and sign flips


@pytest.mark.parametrize("n,depth,n_traj", [(5, 4, 96), (12, 3, 16), (16, 2, 6)])
def test_trajectories_match_oracle(n, depth, n_traj):
    qc = _circuit(n, depth, seed=n)
    ops = lower(qc)
    states, br = run_trajectories(qc, n_traj, seed=100)
    host = states.cpu().numpy()
    checked = 0
    for t in range(n_traj):
        ref, bref, margin = O.noise_trajectory(n, ops, 100 + t)
        if margin < MARGIN:
            continue
        checked += 1
        assert np.array_equal(br[t], bref), t
        assert abs(1 - O.fidelity(host[t], ref)) <= FID_TOL
    assert checked >= n_traj // 2
    assert len(set(map(bytes, br))) > 1          # trajectories differ


@pytest.mark.parametrize("n", [6, 15])
def test_trajectory_alone_equals_batch(n):
    qc = _circuit(n, 3, seed=2)
    states, br = run_trajectories(qc, 8, seed=40)
    for t in (0, 5):
        one, b1 = run_trajectories(qc, 1, seeds=[40 + t])
        assert np.array_equal(one[0].cpu().numpy().view(np.uint32), states[t].cpu().numpy().view(np.uint32))
        assert np.array_equal(b1[0], br[t])


def test_trajectory_average_matches_kraus_density():
    qc = Circuit(3)
    qc.h(0)
    qc.cx(0, 1)
    qc.ry(0.7, 2)
    qc.cx(1, 2)
    qc = add_noise(qc, depolarizing=0.08, amplitude_damping=0.15, dephasing=0.1)
    rho = O.kraus_density(3, lower(qc))
    T = 20000
    states, _ = run_trajectories(qc, T, seed=9, branches=False)
    S = states.cpu().numpy().astype(np.complex128)
    avg = S.T @ S.conj() / T
    assert np.max(np.abs(avg - rho)) < 5 / math.sqrt(T)


def test_noise_only_and_leading_channels():
    # a channel before any gate, and a circuit that is only channels
    qc = Circuit(4)
    qc.amplitude_damp(0.5, 0)
    qc.x(0)
    qc.amplitude_damp(0.5, 0)
    qc.dephase(0.2, 1)
    states, br = run_trajectories(qc, 64, seed=3)
    for t in range(64):
        ref, bref, _ = O.noise_trajectory(4, lower(qc), 3 + t)
        assert np.array_equal(br[t], bref)
        assert np.max(np.abs(states[t].cpu().numpy() - ref)) < 1e-6
    only = Circuit(2)
    only.depolarize(0.9, 1)
    states, br = run_trajectories(only, 32, seed=1)
    for t in range(32):
        ref, bref, _ = O.noise_trajectory(2, lower(only), 1 + t)
        assert np.array_equal(br[t], bref)
        assert np.array_equal(states[t].cpu().numpy(), ref.astype(np.complex64))


def test_unitary_plan_rejects_channels():
    from qsim_b200 import engine as E
    qc = Circuit(3)
    qc.h(0)
    qc.dephase(0.1, 0)
    with pytest.raises(RuntimeError, match="noise channel"):
        E.Plan(3, lower(qc))


def test_simulator_run_samples_noisy_circuit_as_trajectories():
    """BlackwellSimulator.run on a circuit with channels: one trajectory per
    shot, in chunks (14 qubits: 4096 trajectories per chunk, so 5000 shots
    take two)."""
    from blackwell_backend import BlackwellSimulator, HybridSimulator
    qc = Circuit(14, name="decay")
    qc.x(13)
    qc.amplitude_damp(0.3, 13)
    res = BlackwellSimulator().run(qc, shots=5000, seed=4)
    counts = res.get_counts()
    assert sum(counts.values()) == 5000
    assert set(counts) <= {hex(0), hex(1 << 13)}
    n0 = counts.get(hex(0), 0)
    assert 1500 - 4 * 33 < n0 < 1500 + 4 * 33          # P(decay) = 0.3, 4 sigma
    again = BlackwellSimulator().run(qc, shots=5000, seed=4).get_counts()
    assert again == counts                               # seeded trajectories
    hy = HybridSimulator(workers=1, budget_bytes=1 << 30)
    r = hy.run(qc, shots=200, seed=1)
    assert r.metadata["backend_used"] == "blackwell" and sum(r.get_counts().values()) == 200
    hy.close()
