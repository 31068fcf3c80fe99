"""GPU parity of the batch engine, the Chebyshev evolution and the adjoint
gradient."""
import os

import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200 import engine as E
from qsim_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_batch_uneven_widths_vs_oracle_and_alone():
    widths, oo, ops, so = W.qv_batch(40, 4, 17, seed=11)
    bp = E.BatchPlan(widths, oo, ops, so)
    st = bp.alloc_states()
    bp.execute(st)
    torch.cuda.synchronize()
    allv = st.cpu().numpy()
    for c in range(len(widths)):
        n = int(widths[c])
        got = allv[so[c]: so[c] + (1 << n)]
        cops = ops[oo[c]: oo[c + 1]]
        ref = O.simulate(n, cops)
        assert abs(1 - O.fidelity(got, ref)) <= 1e-6, (c, n)
        # alone == in the batch, bit for bit
        alone = E.empty_state(n)
        E.Plan(n, cops).execute_from_zero(alone)
        assert np.array_equal(alone.cpu().numpy(), got), (c, n)


def test_one_shot_batch_slices_equal_batch_plan():
    """qs_batch_run plans a large batch in slices launched as they are ready;
    every state is bit-identical to the reusable plan's, and a bad circuit
    is reported without leaving work queued."""
    widths, oo, ops, so = W.qv_batch(600, 6, 15, seed=12)
    bp = E.BatchPlan(widths, oo, ops, so)
    a = bp.alloc_states()
    bp.execute(a)
    b = torch.full_like(a, 7.0)
    E.batch_run(widths, oo, ops, so, b)
    torch.cuda.synchronize()
    av, bv = a.cpu().numpy(), b.cpu().numpy()
    for c in range(len(widths)):
        n = int(widths[c])
        assert np.array_equal(av[so[c]: so[c] + (1 << n)], bv[so[c]: so[c] + (1 << n)]), c
    for c in (0, 299, 599):
        n = int(widths[c])
        ref = O.simulate(n, ops[oo[c]: oo[c + 1]])
        assert abs(1 - O.fidelity(bv[so[c]: so[c] + (1 << n)], ref)) <= 1e-6
    bad = ops.copy()
    bad["q"][oo[550]][0] = 40                     # qubit out of range in a late slice
    with pytest.raises(Exception):
        E.batch_run(widths, oo, bad, so, b)
    torch.cuda.synchronize()
    E.batch_run(widths, oo, ops, so, b)           # the handle still works
    assert np.array_equal(b.cpu().numpy()[: len(av)], av)


def test_qv8_and_qv4_match_reference_golden():
    import blackwell_kernels as bk
    d = np.load(os.path.join(GOLD, "qv8_ref.npz"))
    probs = bk.qv8_simulate(torch.from_numpy(d["gate_matrices"]), torch.from_numpy(d["gate_qubits"]),
                            d["gate_matrices"].shape[0]).cpu().numpy()
    np.testing.assert_allclose(probs, d["probs"], atol=3e-6)
    d = np.load(os.path.join(GOLD, "qv4_ref.npz"))
    probs = bk.qv4_simulate_cuda(d["gate_data"], d["pair_ids"]).cpu().numpy()
    np.testing.assert_allclose(probs, d["probs"], atol=3e-6)
    np.testing.assert_allclose(bk.heavy_output_probability(probs), d["hop"], atol=1e-5)


def _hams(n):
    from qsim_b200.paulis import PauliSum
    z = PauliSum.from_list([("I" * (n - 1) + "Z", 1.0)])
    heis, tfim = [], []
    for i in range(n - 1):
        for p in "XYZ":
            lab = ["I"] * n
            lab[i] = lab[i + 1] = p
            heis.append(("".join(lab), 0.5))
        lab = ["I"] * n
        lab[i] = lab[i + 1] = "Z"
        tfim.append(("".join(lab), 1.0))
    for i in range(n):
        lab = ["I"] * n
        lab[i] = "X"
        tfim.append(("".join(lab), 1.0))
    return [z, PauliSum.from_list(heis), PauliSum.from_list(tfim)]


@pytest.mark.parametrize("n", [4, 8, 12])
@pytest.mark.parametrize("t", [0.5, 1.0])
def test_chebyshev_vs_expm(n, t):
    """ab_test.py:424-466: Z, Heisenberg, TFIM vs dense scipy expm (FP64)."""
    from blackwell_backend import BlackwellSimulator
    sim = BlackwellSimulator()
    for H in _hams(n):
        sv, info = sim.run_hamiltonian(H, t, precision=1e-12)
        ref = O.expm_evolve(H.to_dense(), O.zero_state(n), t)
        assert abs(1 - O.fidelity(sv, ref)) <= 1e-6, info
        assert O.max_abs_err(sv, ref) < 5e-5


@pytest.mark.parametrize("n", [10, 14])
def test_chebyshev_serving_hamiltonian(n):
    import scipy.sparse as sp
    from blackwell_backend import BlackwellSimulator
    H = W.serving_hamiltonian(n, seed=n)
    psi = W.product_state(n, seed=n + 1)
    t = 3.0
    sv, info = BlackwellSimulator().run_hamiltonian(H, t, initial_state=psi.astype(np.complex64), precision=1e-6)
    ref = O.expm_multiply_evolve(sp.csr_matrix(H.to_dense()) if n <= 10 else _sparse(H), psi, t)
    assert abs(1 - O.fidelity(sv, ref)) <= 1e-6, info


def _sparse(H):
    import scipy.sparse as sp
    from qsim_b200.paulis import csr_from_paulis
    rp, ci, v = csr_from_paulis(H)
    return sp.csr_matrix((v.astype(np.complex128), ci, rp), shape=(1 << H.num_qubits,) * 2)


def test_spmv_and_step_mirrors():
    import blackwell_kernels as bk
    from qsim_b200.paulis import csr_from_paulis
    H = W.serving_hamiltonian(9, seed=1)
    rp, ci, v = csr_from_paulis(H)
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(512) + 1j * rng.standard_normal(512)).astype(np.complex64)
    y0 = (rng.standard_normal(512) + 1j * rng.standard_normal(512)).astype(np.complex64)
    X, Y = torch.from_numpy(x).cuda(), torch.from_numpy(y0).cuda()
    bk.spmv_csr(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda(), X, Y,
                0.7, -0.2, 0.3, 0.1)
    A = _sparse(H)
    want = (0.7 - 0.2j) * (A @ x.astype(np.complex128)) + (0.3 + 0.1j) * y0
    np.testing.assert_allclose(Y.cpu().numpy(), want, atol=1e-5)
    acc = torch.zeros_like(X)
    nxt = torch.empty_like(X)
    bk.chebyshev_step_accum(X, Y, nxt, acc, 0.25, -0.5)
    t = 2 * x - Y.cpu().numpy()
    np.testing.assert_allclose(nxt.cpu().numpy(), t, atol=1e-6)
    np.testing.assert_allclose(acc.cpu().numpy(), (0.25 - 0.5j) * t, atol=1e-6)


def test_adjoint_gradient_vs_fd_and_shift():
    n = 8
    qc, npar = W.efficient_su2(n, reps=2)
    from qsim_b200.circuit import lower
    ops = lower(qc)
    ps = W.random_pauli_observable(n, 24, seed=5)
    rng = np.random.default_rng(3)
    P = rng.uniform(0, 2 * np.pi, (3, npar))
    e, g = E.adjoint_gradient(n, ops, npar, P, ps)
    x, z, c = ps.x, ps.z, ps.real_coefs()
    for b in range(3):
        assert abs(e[b] - O.energy(n, ops, P[b], x, z, c)) < 1e-5
        which = list(range(0, npar, 5))
        shift = O.grad_param_shift(n, ops, P[b], x, z, c, which)
        np.testing.assert_allclose(g[b, which], shift, atol=1e-5)
        fd = O.grad_central_fd(n, ops, P[b], x, z, c, which[:6], h=1e-3)
        # central FD bias for one-parameter entry: f'(sin h/h - 1) ~ -1.7e-7 f'
        np.testing.assert_allclose(g[b, which[:6]], fd, atol=1e-5)


def test_adjoint_multi_tile_vs_shift():
    """14 qubits: the reverse sweep runs in 12-qubit tile passes (4 tiles per
    vector), with CNOT chains, a Toffoli and a CZ whose controls lie outside
    the tile, and a dense two-qubit gate."""
    n = 14
    qc, npar = W.efficient_su2(n, reps=2)
    rng = np.random.default_rng(11)
    m, _ = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))
    qc.unitary(m, [3, 13])
    qc.cz(0, 13)
    qc.ccx(12, 1, 7)
    qc.ry(0.3, 13, param_index=0)      # a parameter used twice
    from qsim_b200.circuit import lower
    ops = lower(qc)
    ps = W.random_pauli_observable(n, 16, seed=7)
    P = rng.uniform(0, 2 * np.pi, (2, npar))
    e, g = E.adjoint_gradient(n, ops, npar, P, ps)
    x, z, c = ps.x, ps.z, ps.real_coefs()
    which = [1, 7, 20, 33, npar - 1]    # parameters used once: exact shift rule
    for b in range(2):
        assert abs(e[b] - O.energy(n, ops, P[b], x, z, c)) < 1e-5
        shift = O.grad_param_shift(n, ops, P[b], x, z, c, which)
        np.testing.assert_allclose(g[b, which], shift, atol=1e-5)
        # parameter 0 enters twice: central differences (bias ~1e-7 relative)
        fd = O.grad_central_fd(n, ops, P[b], x, z, c, [0], h=1e-3)
        np.testing.assert_allclose(g[b, [0]], fd, atol=2e-5)


def test_autograd_function():
    from qsim_b200.autograd import ExpectationFunction
    n = 6
    qc, npar = W.efficient_su2(n, reps=1)
    from qsim_b200.circuit import lower
    ops = lower(qc)
    ps = W.random_pauli_observable(n, 10, seed=8)
    theta = torch.tensor(np.random.default_rng(1).uniform(0, 6.28, (2, npar)), dtype=torch.float64,
                         requires_grad=True)
    E_ = ExpectationFunction.apply(theta, n, ops, ps)
    E_.sum().backward()
    x, z, c = ps.x, ps.z, ps.real_coefs()
    for b in range(2):
        shift = O.grad_param_shift(n, ops, theta[b].detach().numpy(), x, z, c, range(npar))
        np.testing.assert_allclose(theta.grad[b].numpy(), shift, atol=1e-5)


@pytest.mark.parametrize("n", [8, 12])
def test_chebyshev_matrix_free_matches_expm_and_csr(n):
    from blackwell_backend import BlackwellSimulator
    H = W.serving_hamiltonian(n, seed=n, n_pairs=min(20, n))
    psi = W.product_state(n, seed=3).astype(np.complex64)
    sim = BlackwellSimulator()
    a, info = sim.run_hamiltonian(H, 2.0, initial_state=psi, precision=1e-8, method="pauli")
    b, _ = sim.run_hamiltonian(H, 2.0, initial_state=psi, precision=1e-8, method="csr")
    ref = O.expm_evolve(H.to_dense(), psi.astype(np.complex128), 2.0)
    assert abs(1 - O.fidelity(a, ref)) <= 1e-6, info
    assert O.max_abs_err(a, ref) < 5e-5
    assert O.max_abs_err(a, b.astype(np.complex128)) < 5e-5


def test_server_mix_equals_alone():
    """Requests give the same result alone and in a concurrent mix."""
    from qsim_b200.server import CircuitRequest, EvolutionRequest, GradientRequest, Server
    from qsim_b200.circuit import lower
    reqs = []
    for i, w in enumerate([10, 13, 16, 11, 18]):
        reqs.append(CircuitRequest(n_qubits=w, ops=W.qv_ops(w, w, 100 + i), shots=512, seed=i))
    qc, npar = W.efficient_su2(8, reps=2)
    obs = W.random_pauli_observable(8, 20, seed=1)
    P = np.random.default_rng(0).uniform(0, 6.28, (2, npar))
    reqs.append(GradientRequest(n_qubits=8, ops=lower(qc), n_params=npar, params=P, observable=obs))
    reqs.append(EvolutionRequest(hamiltonian=W.serving_hamiltonian(10, 4, 10), t=1.5,
                                 psi0=W.product_state(10, 5), precision=1e-8))
    alone = []
    for r in reqs:
        s = Server(workers=1, batch_window_s=0)
        alone.append(s.submit(r).result(120))
        s.close()
    s = Server(workers=4)
    futs = [s.submit(r) for r in reqs]
    mixed = [f.result(120) for f in futs]
    st = s.stats()
    s.close()
    for a, m in zip(alone[:5], mixed[:5]):
        assert np.array_equal(a, m)
    assert np.array_equal(alone[5][0], mixed[5][0]) and np.array_equal(alone[5][1], mixed[5][1])
    assert np.array_equal(alone[6][0], mixed[6][0])
    assert st["completed"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0


def test_batch_plan_graph_replay():
    """A reusable batch plan is captured into a CUDA graph at its second
    execution and replayed afterwards; every execution gives the same bits,
    also after switching to another states buffer (re-capture)."""
    widths, oo, ops, so = W.qv_batch(24, 6, 16, seed=21)
    bp = E.BatchPlan(widths, oo, ops, so)
    a = bp.alloc_states()
    b = bp.alloc_states()
    runs = []
    for buf in (a, a, a, b, b, a):
        buf.zero_()
        bp.execute(buf)
        torch.cuda.synchronize()
        runs.append(buf.cpu().numpy().copy())
    for r in runs[1:]:
        assert np.array_equal(runs[0], r)
    c = 3
    n = int(widths[c])
    ref = O.simulate(n, ops[oo[c]: oo[c + 1]])
    assert abs(1 - O.fidelity(runs[-1][so[c]: so[c] + (1 << n)], ref)) <= 1e-6


def test_autotune_widths_then_alone_equals_batch():
    """The autotuner records one (tile, block) shape per width; batches and
    single-circuit plans then share it, so results agree bit for bit."""
    widths, oo, ops, so = W.qv_batch(30, 10, 17, seed=31)
    try:
        table = E.autotune_batch(widths, oo, ops)
        assert set(table) == {int(w) for w in widths}
        for w, (tb, bb) in table.items():
            assert 2 <= bb <= 5 and (w <= 14 or 12 <= tb <= 14)
        bp = E.BatchPlan(widths, oo, ops, so)
        st = bp.alloc_states()
        bp.execute(st)
        torch.cuda.synchronize()
        allv = st.cpu().numpy()
        for c in range(0, len(widths), 3):
            n = int(widths[c])
            got = allv[so[c]: so[c] + (1 << n)]
            assert abs(1 - O.fidelity(got, O.simulate(n, ops[oo[c]: oo[c + 1]]))) <= 1e-6
            alone = E.empty_state(n)
            E.Plan(n, ops[oo[c]: oo[c + 1]]).execute_from_zero(alone)
            assert np.array_equal(alone.cpu().numpy(), got), (c, n)
    finally:
        E.autotune_clear()


def test_adjoint_per_gate_fallback_agrees(tmp_path):
    """The one-launch-per-gate sweep (used past 1 GiB of pass partials, or
    with QSIM_ADJ_PASSES=0) gives the same gradients as the tile passes."""
    import os
    import subprocess
    import sys
    ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = r"""
import sys, numpy as np
sys.path[:0] = %r
from qsim_b200 import engine as E, workloads as W
from qsim_b200.circuit import lower
qc, npar = W.efficient_su2(14, reps=2)
qc.cz(0, 13)
ops = lower(qc)
ps = W.random_pauli_observable(14, 12, seed=3)
P = np.random.default_rng(2).uniform(0, 6.28, (2, npar))
e, g = E.adjoint_gradient(14, ops, npar, P, ps)
np.save(sys.argv[1], np.concatenate([e, g.ravel()]))
""" % ([os.path.join(ROOT, "qiskit-blackwell_b200", "python"), os.path.join(ROOT, "oracle")],)
    out = {}
    for flag in ("1", "0"):
        path = str(tmp_path / f"adj_{flag}.npy")
        env = dict(os.environ, QSIM_ADJ_PASSES=flag)
        subprocess.run([sys.executable, "-c", code, path], env=env, check=True, timeout=300)
        out[flag] = np.load(path)
    np.testing.assert_allclose(out["1"], out["0"], atol=1e-6)


def test_batch_is_one_persistent_launch_with_bounded_waits():
    """A batch plan runs as one persistent launch (tiles taken from a device
    counter level by level, each state's next pass waiting for its previous
    one).  With one pass of one state left uncounted (the wait-test hook),
    the dependent waits run out after 50 ms, the status word reports them,
    and the next execution is complete and right."""
    import ctypes as C
    widths, oo, ops, so = W.qv_batch(24, 14, 18, seed=41)
    h = E._h()
    h.call("qs_set_batch_queue", 1)
    try:
        bp = E.BatchPlan(widths, oo, ops, so)
    finally:
        h.call("qs_set_batch_queue", 0)
    assert bp.info["n_launches"] == 1 and bp.info["max_passes"] >= 2
    st = bp.alloc_states()
    code = C.c_int(-1)
    h.call("qs_device_status", C.byref(code))
    assert code.value == 0
    l0 = h.launches()
    bp.execute(st)
    torch.cuda.synchronize()
    assert h.launches() - l0 == 1
    h.call("qs_set_wait_test", 2)
    bp.execute(st)
    torch.cuda.synchronize()
    h.call("qs_device_status", C.byref(code))
    assert code.value == 4, code.value
    st.zero_()
    bp.execute(st)
    torch.cuda.synchronize()
    h.call("qs_device_status", C.byref(code))
    assert code.value == 0
    allv = st.cpu().numpy()
    for c in range(len(widths)):
        n = int(widths[c])
        got = allv[so[c]: so[c] + (1 << n)]
        assert abs(1 - O.fidelity(got, O.simulate(n, ops[oo[c]: oo[c + 1]]))) <= 1e-6, c
    # the per-level launches give the same bits (on the CUDA cores, as the
    # persistent launch runs every pass)
    h.call("qs_set_tensor_cores", 0)
    try:
        bl = E.BatchPlan(widths, oo, ops, so)
    finally:
        h.call("qs_set_tensor_cores", 1)
    assert bl.info["n_launches"] > 1
    st2 = bl.alloc_states()
    bl.execute(st2)
    torch.cuda.synchronize()
    assert np.array_equal(st2.cpu().numpy().view(np.uint32), allv.view(np.uint32))
