"""GPU parity of the planner + fused tile-pass kernel (the plain per-circuit
path) against the FP64 oracle: |1-F| <= 1e-6 and a max-amplitude bound."""
import math

import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200 import engine as E
from qsim_b200 import workloads as W
from qsim_b200.circuit import Circuit, lower
from test_oracle_golden import _random_ops

pytestmark = pytest.mark.gpu


def amp_bound(n_ops):
    # FP32 FMA chains: each dense op adds at most a few ulps per amplitude;
    # the bound is stated per op on a normalised state.
    return 2e-7 * max(n_ops, 1) ** 0.5 * 8


def run_plan(n, ops, from_zero=True, psi0=None):
    plan = E.Plan(n, ops)
    s = E.empty_state(n)
    if from_zero:
        plan.execute_from_zero(s)
    else:
        s.copy_(torch.from_numpy(psi0.astype(np.complex64)))
        plan.execute(s)
    torch.cuda.synchronize()
    return s.cpu().numpy(), plan.info


def test_config0_qv12_through_backend():
    from blackwell_backend import BlackwellSimulator
    ops = W.qv_ops(12, 12, 0)
    qc = Circuit(12, name="qv12")
    for r in ops:
        qc.unitary((r["m"][0:32:2] + 1j * r["m"][1:32:2]).reshape(4, 4), [int(r["q"][0]), int(r["q"][1])])
    sv, _ = BlackwellSimulator().run_statevector(qc)
    ref = O.simulate(12, ops)
    assert abs(1 - O.fidelity(sv, ref)) <= 1e-6
    assert O.max_abs_err(sv, ref) <= amp_bound(72)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 9, 13, 14, 15, 17])
def test_random_all_kinds(n):
    rng = np.random.default_rng(1000 + n)
    ops = _random_ops(n, 120, rng)
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi0 = (psi0 / np.linalg.norm(psi0)).astype(np.complex64)
    sv, info = run_plan(n, ops, from_zero=False, psi0=psi0)
    ref = O.simulate(n, ops, psi0.astype(np.complex128))
    assert abs(1 - O.fidelity(sv, ref)) <= 1e-6, info
    assert O.max_abs_err(sv, ref) <= amp_bound(120), info


@pytest.mark.parametrize("tile_bits", [10, 12, 13, 14])
def test_multipass_layers_20q(tile_bits):
    """The 32-qubit layer generator at 20 qubits: many passes."""
    from qsim_b200 import _lib
    h = E._h()
    h.call("qs_set_tile_bits", tile_bits)
    try:
        ops = W.layers_ops(20, 8, seed=3)
        sv, info = run_plan(20, ops)
        assert info["n_passes"] > 1
        ref = O.simulate(20, ops)
        assert abs(1 - O.fidelity(sv, ref)) <= 1e-6
        assert O.max_abs_err(sv, ref) <= amp_bound(len(ops))
    finally:
        h.call("qs_set_tile_bits", 0)


def test_config1_generator_fidelity_26q():
    """Config-1 generator (20 layers, Toffolis) checked against FP64 at 26 qubits."""
    ops = W.layers_ops(26, 20, seed=0)
    sv, info = run_plan(26, ops)
    ref = O.simulate(26, ops)
    assert abs(1 - O.fidelity(sv, ref)) <= 1e-6, info
    assert O.max_abs_err(sv, ref) <= 1e-5


def test_analytic_pins():
    """tests/stress_test.py pins: GHZ, uniform superposition, H^1000=I, X^999,
    CX^1000, Rz accumulation, 500 x Rx(2pi/500) back to |0>."""
    from blackwell_backend import BlackwellSimulator
    sim = BlackwellSimulator()
    n = 16
    qc = Circuit(n)
    qc.h(0)
    for q in range(n - 1):
        qc.cx(q, q + 1)
    sv, _ = sim.run_statevector(qc)
    p = np.abs(sv) ** 2
    assert abs(p[0] - 0.5) < 1e-6 and abs(p[-1] - 0.5) < 1e-6 and p[1:-1].sum() < 1e-10
    qc = Circuit(n)
    for q in range(n):
        qc.h(q)
    sv, _ = sim.run_statevector(qc)
    assert np.max(np.abs(np.abs(sv) - 2 ** (-n / 2))) < 1e-6
    qc = Circuit(8)
    for _ in range(1000):
        qc.h(3)
    sv, _ = sim.run_statevector(qc)
    assert abs(abs(sv[0]) - 1) < 1e-5
    qc = Circuit(8)
    for _ in range(999):
        qc.x(5)
    sv, _ = sim.run_statevector(qc)
    assert sv[1 << 5] == 1
    qc = Circuit(8)
    qc.h(2)
    for _ in range(1000):
        qc.cx(2, 6)
    sv, _ = sim.run_statevector(qc)
    assert abs(abs(sv[0]) ** 2 - 0.5) < 1e-6 and abs(abs(sv[4]) ** 2 - 0.5) < 1e-6
    qa, qb = Circuit(8), Circuit(8)
    qa.h(4)
    qb.h(4)
    for _ in range(1000):
        qa.rz(math.pi / 3 / 1000, 4)
    qb.rz(math.pi / 3, 4)
    a, _ = sim.run_statevector(qa)
    b, _ = sim.run_statevector(qb)
    assert abs(np.vdot(a, b)) ** 2 > 1 - 1e-6
    qc = Circuit(8)
    for _ in range(500):
        qc.rx(2 * math.pi / 500, 7)
    sv, _ = sim.run_statevector(qc)
    assert abs(abs(sv[0]) - 1) < 1e-4 and np.max(np.abs(sv[1:])) < 1e-4


def test_plan_determinism_and_reuse():
    ops = W.qv_ops(18, 18, 4)
    plan = E.Plan(18, ops)
    a = E.empty_state(18)
    b = E.empty_state(18)
    plan.execute_from_zero(a)
    plan.execute_from_zero(b)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_measure_reset_midcircuit():
    from blackwell_backend import BlackwellSimulator
    sim = BlackwellSimulator()
    qc = Circuit(3, 1)
    qc.x(0).measure(0, 0).reset(0).h(1)
    sv, _ = sim.run_statevector(qc)
    ref = np.zeros(8, dtype=complex)
    ref[0] = ref[2] = 2 ** -0.5
    assert np.max(np.abs(sv - ref)) < 1e-6
