"""GPU parity at the benchmark configurations' real sizes.

* Batching (4096 Quantum-Volume circuits, widths 10-20): 96 circuits of the
  same generator through the autotuner and a batch plan, every circuit
  against the FP64 oracle and bit for bit against the same circuit alone;
  then once more with 14-qubit tiles forced, the shape the autotuner picks
  for widths 18-19 (one CTA per SM, the twice-the-threads pass kernel).
* Differentiation (20-qubit EfficientSU2, 4 reps, 200 parameters, 256-term
  observable): energies of 4 parameter vectors against the FP64 oracle, and
  the adjoint gradient against the parameter-shift rule on 20 seeded
  parameters and against central differences (h = 1e-3) on 5 of them.
* Serving: a 22-qubit gradient, a 22-qubit Chebyshev evolution and a
  24-qubit QV circuit, each the same alone and in a mix with smaller
  requests; the evolution against scipy's expm_multiply (FP64), the gradient
  against the oracle's energy and parameter shift, the QV circuit's state
  against the oracle and its shots against the oracle's distribution.

Tolerances: |1-F| <= 1e-6 against FP64 for states, 1e-5 for gradients and
energies (absolute), bit-identical where the same kernels run the same plan.
"""
import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200 import engine as E
from qsim_b200 import workloads as W
from qsim_b200.circuit import lower

pytestmark = pytest.mark.gpu


def _check_batch(widths, oo, ops, so, refs):
    bp = E.BatchPlan(widths, oo, ops, so)
    st = bp.alloc_states()
    bp.execute(st)
    torch.cuda.synchronize()
    allv = st.cpu().numpy()
    worst = 0.0
    for c in range(len(widths)):
        n = int(widths[c])
        got = allv[so[c]: so[c] + (1 << n)]
        cops = ops[oo[c]: oo[c + 1]]
        err = abs(1 - O.fidelity(got, refs[c]))
        worst = max(worst, err)
        assert err <= 1e-6, (c, n, err)
        alone = E.empty_state(n)
        E.Plan(n, cops).execute_from_zero(alone)
        assert np.array_equal(alone.cpu().numpy(), got), (c, n)
    return worst, bp.info


def test_qv_batch_widths_10_to_20_autotuned_and_14_bit_tiles():
    widths, oo, ops, so = W.qv_batch(96, 10, 20, seed=1)
    assert {18, 19, 20} <= set(int(w) for w in widths)
    refs = [O.simulate(int(widths[c]), ops[oo[c]: oo[c + 1]]) for c in range(len(widths))]
    h = E._h()
    try:
        table = E.autotune_batch(widths, oo, ops)
        assert set(table) == set(int(w) for w in widths)
        _check_batch(widths, oo, ops, so, refs)
        # the 14-qubit tile shape on every width (2x-thread CTAs, one per SM)
        E.autotune_clear()
        h.call("qs_set_tile_bits", 14)
        h.call("qs_set_block_bits", 5)
        _, info = _check_batch(widths, oo, ops, so, refs)
        assert info["n_items"] > 0
    finally:
        h.call("qs_set_tile_bits", 0)
        h.call("qs_set_block_bits", 0)
        E.autotune_clear()


def test_adjoint_config3_full_size():
    n = 20
    qc, npar = W.efficient_su2(n, reps=4)
    assert npar == 200
    ops = lower(qc)
    ps = W.random_pauli_observable(n, 256, seed=7)
    rng = np.random.default_rng(3)
    P = rng.uniform(0, 2 * np.pi, (4, npar))
    e, g = E.adjoint_gradient(n, ops, npar, P, ps)
    x, z, c = ps.x, ps.z, ps.real_coefs()
    for b in range(4):
        assert abs(e[b] - O.energy(n, ops, P[b], x, z, c)) < 1e-5, b
    which = sorted(np.random.default_rng(9).choice(npar, 20, replace=False).tolist())
    shift = O.grad_param_shift(n, ops, P[0], x, z, c, which)
    np.testing.assert_allclose(g[0, which], shift, atol=1e-5)
    # every parameter enters once: central differences are biased by
    # f'(sin h / h - 1) ~ -1.7e-7 f', far inside the tolerance
    fd = O.grad_central_fd(n, ops, P[0], x, z, c, which[:5], h=1e-3)
    np.testing.assert_allclose(g[0, which[:5]], fd, atol=1e-5)


def _sparse64(H):
    import scipy.sparse as sp
    from qsim_b200.paulis import csr_from_paulis
    rp, ci, v = csr_from_paulis(H)
    return sp.csr_matrix((v.astype(np.complex128), ci, rp), shape=(1 << H.num_qubits,) * 2)


def test_serving_mix_22_and_24_qubits_alone_equals_mixed():
    from qsim_b200.server import CircuitRequest, EvolutionRequest, GradientRequest, NativeServer
    qc, npar = W.efficient_su2(22, reps=4)
    obs = W.random_pauli_observable(22, 256, seed=22)
    P = np.random.default_rng(1).uniform(0, 2 * np.pi, (1, npar))
    H = W.serving_hamiltonian(22, seed=22)
    psi0 = W.product_state(22, seed=23)
    t = 0.5
    big = [
        CircuitRequest(n_qubits=24, ops=W.qv_ops(24, 24, 1_000_024), shots=1024, seed=24),
        GradientRequest(n_qubits=22, ops=lower(qc), n_params=npar, params=P, observable=obs),
        EvolutionRequest(hamiltonian=H, t=t, psi0=psi0, precision=1e-6),
    ]
    small = [CircuitRequest(n_qubits=w, ops=W.qv_ops(w, w, 500 + i), shots=256, seed=i)
             for i, w in enumerate([10, 14, 17, 12, 19])]
    reqs = big + small
    alone = []
    for r in reqs:
        s = NativeServer(workers=1)
        alone.append(s.submit(r).result(600))
        s.close()
    s = NativeServer(workers=4)
    futs = [s.submit(r) for r in reqs]
    mixed = [f.result(600) for f in futs]
    st = s.stats()
    s.close()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert np.array_equal(alone[0], mixed[0])
    assert np.array_equal(alone[1][0], mixed[1][0]) and np.array_equal(alone[1][1], mixed[1][1])
    assert np.array_equal(alone[2][0], mixed[2][0])
    for k in range(3, len(reqs)):
        assert np.array_equal(alone[k], mixed[k]), k

    # 24-qubit QV: the batch engine's state (the kernels the server runs) vs
    # FP64, and the served shots against the oracle's distribution: for a
    # Porter-Thomas distribution E[N p(x)] = N sum p^2 ~ 2, uniform shots give 1
    qv = big[0]
    st24 = torch.empty(1 << 24, dtype=torch.complex64, device="cuda")
    E.batch_run(np.array([24], np.int32), np.array([0, len(qv.ops)], np.int64), qv.ops,
                np.array([0], np.int64), st24)
    ref = O.simulate(24, qv.ops)
    assert abs(1 - O.fidelity(st24.cpu().numpy(), ref)) <= 1e-6
    p = np.abs(ref) ** 2
    shots = np.asarray(mixed[0], dtype=np.int64)
    assert shots.shape == (1024,) and shots.min() >= 0 and shots.max() < (1 << 24)
    stat = float(np.mean(p[shots])) * (1 << 24)
    assert 1.6 < stat < 2.5, stat

    # 22-qubit gradient: energy vs FP64 and 4 parameter-shift entries
    g = big[1]
    x, z, c = obs.x, obs.z, obs.real_coefs()
    assert abs(mixed[1][0][0] - O.energy(22, g.ops, P[0], x, z, c)) < 1e-5
    which = [0, 57, 123, npar - 1]
    shift = O.grad_param_shift(22, g.ops, P[0], x, z, c, which)
    np.testing.assert_allclose(np.asarray(mixed[1][1])[0, which], shift, atol=1e-5)

    # 22-qubit evolution vs expm_multiply in FP64
    ref = O.expm_multiply_evolve(_sparse64(H), psi0.astype(np.complex128), t)
    got = np.asarray(mixed[2][0])
    assert abs(1 - O.fidelity(got, ref)) <= 1e-6
