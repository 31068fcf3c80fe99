"""The native serving runtime (qs_server_* in the C ABI) through its Python
wrapper: results equal the same requests run alone and the direct engine
calls; admission, cancellation and deadlines are reported per request."""
import time

import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200 import engine as E
from qsim_b200 import workloads as W
from qsim_b200.circuit import lower
from qsim_b200.server import (AdmissionError, Cancelled, CircuitRequest, DeadlineExceeded, EvolutionRequest,
                              GradientRequest, NativeServer)

pytestmark = pytest.mark.gpu


def _requests():
    reqs = [CircuitRequest(n_qubits=w, ops=W.qv_ops(w, w, 300 + i), shots=512, seed=i)
            for i, w in enumerate([10, 13, 16, 11, 18, 12])]
    qc, npar = W.efficient_su2(8, reps=2)
    obs = W.random_pauli_observable(8, 20, seed=1)
    P = np.random.default_rng(0).uniform(0, 6.28, (2, npar))
    reqs.append(GradientRequest(n_qubits=8, ops=lower(qc), n_params=npar, params=P, observable=obs))
    reqs.append(EvolutionRequest(hamiltonian=W.serving_hamiltonian(10, 4, 10), t=1.5,
                                 psi0=W.product_state(10, 5), precision=1e-8))
    return reqs


def test_native_mix_equals_alone_and_engine():
    reqs = _requests()
    alone = []
    for r in reqs:
        s = NativeServer(workers=1)
        alone.append(s.submit(r).result(120))
        s.close()
    s = NativeServer(workers=4)
    futs = [s.submit(r) for r in reqs]
    mixed = [f.result(120) for f in futs]
    st = s.stats()
    s.close()
    for a, m in zip(alone[:6], mixed[:6]):
        assert np.array_equal(a, m)
    assert np.array_equal(alone[6][0], mixed[6][0]) and np.array_equal(alone[6][1], mixed[6][1])
    assert np.array_equal(alone[7][0], mixed[7][0])
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["p99_ms"] >= st["p50_ms"] > 0
    # circuits: samples follow the exact distribution (chi-square-free check on
    # the most likely outcome) and stay inside the state
    for r, smp in zip(reqs[:6], mixed[:6]):
        assert smp.shape == (512,) and smp.min() >= 0 and smp.max() < (1 << r.n_qubits)
    # gradient and evolution equal the direct engine calls bit for bit
    g = reqs[6]
    e_ref, g_ref = E.adjoint_gradient(g.n_qubits, g.ops, g.n_params, g.params, g.observable)
    assert np.array_equal(e_ref, mixed[6][0]) and np.array_equal(g_ref, mixed[6][1])
    ev = reqs[7]
    from blackwell_backend.chebyshev import chebyshev_evolve_pauli
    psi = torch.as_tensor(np.asarray(ev.psi0, dtype=np.complex64)).cuda()
    out, _ = chebyshev_evolve_pauli(psi, ev.hamiltonian, ev.t, precision=ev.precision)
    assert np.array_equal(out.cpu().numpy(), mixed[7][0])


def test_native_sampling_distribution():
    """A Bell-like circuit: only |0..0> and |1..1>, about half each."""
    n = 12
    recs = []
    from qsim_b200.circuit import Circuit
    qc = Circuit(n)
    qc.h(0)
    for q in range(1, n):
        qc.cx(0, q)
    ops = lower(qc)
    s = NativeServer(workers=2)
    smp = s.submit(CircuitRequest(n_qubits=n, ops=ops, shots=4000, seed=7)).result(60)
    s.close()
    assert set(np.unique(smp)) <= {0, (1 << n) - 1}
    assert 1700 < int((smp == 0).sum()) < 2300


def test_native_admission_cancel_deadline():
    s = NativeServer(budget_bytes=1 << 26, workers=1)   # 64 MiB
    try:
        big = s.submit(CircuitRequest(n_qubits=24, ops=W.qv_ops(24, 2, 1), shots=1, seed=0))  # 128 MiB
        with pytest.raises(AdmissionError):
            big.result(10)
        # occupy the single worker, then queue requests behind it
        blocker = s.submit(CircuitRequest(n_qubits=22, ops=W.qv_ops(22, 22, 2), shots=1, seed=0))
        late = s.submit(CircuitRequest(n_qubits=22, ops=W.qv_ops(22, 4, 3), shots=1, seed=0, deadline_s=1e-6))
        queued = s.submit(CircuitRequest(n_qubits=22, ops=W.qv_ops(22, 4, 4), shots=1, seed=0))
        cancelled = s.cancel(queued)
        blocker.result(60)
        with pytest.raises((DeadlineExceeded, Cancelled)):
            late.result(60)
        if cancelled:
            with pytest.raises(Cancelled):
                queued.result(60)
        else:   # it was admitted before the cancel arrived
            queued.result(60)
        st = s.stats()
        assert st["completed"] >= 1 and st["budget_bytes"] == 1 << 26
    finally:
        s.close()
