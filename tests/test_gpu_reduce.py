"""GPU parity of the FP64 reductions: norm, renormalise, probabilities,
measurement, sampling and Pauli expectations; determinism."""
import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200 import engine as E
from qsim_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rand_state(n, seed, norm=1.0):
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return (norm * psi / np.linalg.norm(psi)).astype(np.complex64)


@pytest.mark.parametrize("n", [1, 4, 12, 20, 23])
def test_norm_probs_renorm(n):
    psi = rand_state(n, n, norm=1.3)
    s = torch.from_numpy(psi).cuda()
    ref = np.sum(np.abs(psi.astype(np.complex128)) ** 2)
    assert abs(E.norm2(s) - ref) <= 1e-12 * max(1.0, ref) * 64
    p = E.probs(s).cpu().numpy()
    np.testing.assert_allclose(p, np.abs(psi) ** 2, rtol=1e-6, atol=1e-12)
    E.renormalize(s)
    assert abs(E.norm2(s) - 1.0) < 1e-6


def test_measure_matches_oracle():
    n = 10
    psi = rand_state(n, 3)
    p0 = {t: float(np.sum(np.abs(psi.astype(np.complex128).reshape(-1)[((np.arange(1 << n) >> t) & 1) == 0]) ** 2))
          for t in range(n)}
    for t in range(n):
        for u, want in ((p0[t] - 1e-4, 0), (p0[t] + 1e-4, 1)):
            s = torch.from_numpy(psi.copy()).cuda()
            out = E.measure(s, t, u)
            assert out == want
            v = s.cpu().numpy().astype(np.complex128)
            keep = ((np.arange(1 << n) >> t) & 1) == want
            exp = np.where(keep, psi, 0) / np.sqrt(p0[t] if want == 0 else 1 - p0[t])
            assert np.max(np.abs(v - exp)) < 1e-6


@pytest.mark.parametrize("n", [3, 11, 18])
def test_sample_matches_oracle(n):
    psi = rand_state(n, 40 + n)
    s = torch.from_numpy(psi).cuda()
    rng = np.random.default_rng(n)
    u = rng.uniform(0, 1, 20000)
    u = np.concatenate([u, [0.0, 1.0, 1.5, 1e-300]])
    cdf = np.cumsum(np.abs(psi.astype(np.complex128)) ** 2)
    # drop draws within 1e-12 of a CDF step (FP64 summation-order ties)
    near = np.min(np.abs(cdf[None, :] - u[:, None]), axis=1) < 1e-12 if n <= 11 else np.zeros(u.size, bool)
    u = u[~near]
    got = E.sample_u(s, torch.from_numpy(u).cuda()).cpu().numpy()
    want = O.sample_indices(psi.astype(np.complex128), u)
    assert np.array_equal(got, want)


def test_sample_counts_statistics():
    """Bell state: no spurious outcomes (stress_test.py:545-569); 50k-shot
    chi-square on a skewed state (stress_test.py:519-543)."""
    import blackwell_kernels as bk
    s = bk.state_init(2)
    bk.apply_gate(s, bk.hadamard_gate(), 0)
    bk.apply_mcgate(s, bk.pauli_x_gate(), [0], 1)
    torch.manual_seed(0)
    out = bk.sample(s, 20000).cpu().numpy()
    assert set(np.unique(out)) <= {0, 3}
    assert abs(np.mean(out == 0) - 0.5) < 0.02


def test_expectations_match_oracle():
    import blackwell_kernels as bk
    n = 12
    psi = rand_state(n, 9)
    s = torch.from_numpy(psi).cuda()
    p128 = psi.astype(np.complex128)
    for zm in (0, 1, 0b101, (1 << n) - 1):
        assert abs(bk.expectation_z(s, zm) - O.pauli_expectation(p128, [0], [zm], [1.0])) < 1e-6
    for q in (0, 5, 11):
        for opk in (1, 2):
            zm = 0b10010 & ~(1 << q)
            x = 1 << q
            z = zm | (x if opk == 2 else 0)
            assert abs(bk.expectation_pauli(s, zm, q, opk) - O.pauli_expectation(p128, [x], [z], [1.0])) < 1e-6
    ps = W.random_pauli_observable(n, 64, seed=2)
    got = E.expect_pauli_sum(s, ps)
    want = O.pauli_expectation(p128, ps.x, ps.z, ps.real_coefs())
    assert abs(got - want) < 1e-5 * max(1, abs(want))
    # determinism: bit-identical on repeat
    assert E.expect_pauli_sum(s, ps) == got
    hpsi = E.apply_pauli_sum(s, ps).cpu().numpy()
    H = ps.to_dense()
    np.testing.assert_allclose(hpsi, H @ p128, atol=2e-5)
