"""Sampler/Estimator wrappers and the device-side counts histogram."""
import numpy as np
import pytest

import sv_oracle as O
from qsim_b200 import workloads as W
from qsim_b200.circuit import Circuit

pytestmark = pytest.mark.gpu


def _ghz(n):
    qc = Circuit(n, name=f"ghz{n}")
    qc.h(0)
    for q in range(1, n):
        qc.cx(q - 1, q)
    return qc


def test_sampler_counts_on_device():
    from blackwell_backend.primitives import Sampler
    res = Sampler().run([_ghz(5), _ghz(9)], shots=2000, seed=3)
    for n, counts in zip((5, 9), res):
        assert set(counts) <= {hex(0), hex((1 << n) - 1)}
        assert sum(counts.values()) == 2000
        assert 850 < counts.get(hex(0), 0) < 1150


def test_estimator_matches_oracle():
    from blackwell_backend.primitives import Estimator
    from qsim_b200.circuit import lower
    qc = _ghz(6)
    obs = [("ZZIIII", 1.0), ("XXXXXX", 0.5), ("IIIYYI", -0.25)]
    val = Estimator().run([(qc, obs)])[0]
    # <GHZ|Z5 Z4|GHZ> = 1, <X^6> = 1, <Y2 Y1> = 0 (labels: leftmost = highest qubit)
    assert abs(val - 1.5) < 1e-6
    ps = W.random_pauli_observable(6, 20, seed=2)
    qc2 = Circuit(6)
    for q in range(6):
        qc2.ry(0.3 + 0.2 * q, q)
    qc2.cx(0, 5)
    v2 = Estimator().run([(qc2, ps)])[0]
    psi = O.simulate(6, lower(qc2))
    assert abs(v2 - O.pauli_expectation(psi, ps.x, ps.z, ps.real_coefs())) < 1e-6


def test_primitives_on_noisy_circuits():
    """Sampler: one trajectory per shot; Estimator: the trajectory mean of
    <H>, against Tr(rho H) from the oracle's Kraus-sum density matrix."""
    from blackwell_backend.primitives import Estimator, Sampler
    from qsim_b200.circuit import lower
    from qsim_b200.noise import add_noise
    qc = Circuit(3, name="noisy3")
    qc.h(0)
    qc.cx(0, 1)
    qc.ry(0.7, 2)
    qc = add_noise(qc, depolarizing=0.05, amplitude_damping=0.2, dephasing=0.1)
    counts = Sampler().run([qc], shots=3000, seed=2)[0]
    assert sum(counts.values()) == 3000
    rho = O.kraus_density(3, lower(qc))
    obs = [("ZII", 1.0), ("IZZ", 0.5), ("XXI", -0.25)]
    zi = np.diag([1, 1, 1, 1, -1, -1, -1, -1]).astype(complex)          # Z on qubit 2 (leftmost label)
    z = np.diag([1, -1]).astype(complex)
    x = np.array([[0, 1], [1, 0]], dtype=complex)
    i2 = np.eye(2)
    H = 1.0 * np.kron(np.kron(z, i2), i2) + 0.5 * np.kron(np.kron(i2, z), z) - 0.25 * np.kron(np.kron(x, x), i2)
    exact = float(np.real(np.trace(rho @ H)))
    T = 20000
    val = Estimator(trajectories=T, seed=5).run([(qc, obs)])[0]
    assert abs(val - exact) < 5 * 1.75 / np.sqrt(T)                      # |H| <= 1.75, 5 sigma
    assert np.allclose(zi, np.kron(np.kron(z, i2), i2))
