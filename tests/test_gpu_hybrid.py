"""HybridSimulator on the GPU: every route gives the same counts for the same
seed (the plan, the batch plan and the serving runtime compute identical
states and draw identical uniforms), lists are split by the policy, and the
route log / metadata follow the reference's shapes (hybrid.py:177-286)."""
import numpy as np
import pytest

import sv_oracle as O
from qsim_b200.circuit import Circuit, lower

pytestmark = pytest.mark.gpu


def _qv(n, seed, name=None, measure=True):
    rng = np.random.default_rng(seed)
    qc = Circuit(n, n, name=name or f"qv{n}_{seed}")
    for _ in range(n):
        perm = rng.permutation(n)
        for k in range(0, n - 1, 2):
            m, _ = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))
            qc.unitary(m, [int(perm[k]), int(perm[k + 1])])
    if measure:
        for q in range(n):
            qc.measure(q, q)
    return qc


@pytest.fixture(scope="module")
def sim():
    from blackwell_backend.hybrid import HybridSimulator
    s = HybridSimulator(workers=2, budget_bytes=4 << 30)
    yield s
    s.close()


def test_routes_give_identical_counts(sim):
    qc = _qv(11, 4)
    res = {r: sim.run(qc, shots=3000, seed=99, backend=r) for r in ("blackwell", "batched", "served")}
    counts = {r: v.get_counts() for r, v in res.items()}
    assert counts["blackwell"] == counts["batched"] == counts["served"]
    assert sum(counts["served"].values()) == 3000
    for r, v in res.items():
        assert v.metadata["backend_used"] == r
        assert v.metadata["analysis"]["non_native_ratio"] > 0.5


def test_statevector_routes_bit_identical_and_match_oracle(sim):
    qc = _qv(9, 5, measure=False)
    sv_a, _, ra = sim.run_statevector(qc, backend="blackwell")
    sv_b, _, rb = sim.run_statevector(qc, backend="batched")
    assert (ra, rb) == ("blackwell", "batched")
    assert np.array_equal(sv_a.view(np.uint32), sv_b.view(np.uint32))
    ref = O.simulate(9, lower(qc))
    assert abs(1.0 - O.fidelity(sv_a, ref)) <= 1e-6
    both = sim.run_both(qc)
    assert abs(both["fidelity"] - 1.0) < 1e-9
    assert set(both) >= {"blackwell_sv", "batched_sv", "blackwell_time_ms", "batched_time_ms", "speedup"}


def test_list_routing_and_alone_equals_list(sim):
    from blackwell_backend.hybrid import HybridSimulator, RoutingPolicy
    circs = [_qv(w, 10 + w) for w in (6, 8, 10, 12)]
    wide = Circuit(21, name="wide21")
    wide.h(20)
    wide.cx(20, 0)
    circs.append(wide)                                   # wider than batch_max_qubits
    n0 = len(sim.route_log)
    res = sim.run(circs, shots=500, seed=7)
    log = sim.route_log[n0:]
    used = {e["circuit_name"]: e["backend_used"] for e in log}
    assert used["wide21"] == "blackwell"
    assert all(used[c.name] == "batched" for c in circs[:4])
    assert all(e["success"] for e in log)
    for k, (c, r) in enumerate(zip(circs, res)):
        alone = sim.run(c, shots=500, seed=7 + k, backend="blackwell")
        assert r.get_counts() == alone.get_counts(), c.name
    wc = res[-1].get_counts()
    assert set(wc) <= {hex(0), hex((1 << 20) | 1)}


def test_submit_futures_and_forced_served(sim):
    futs = [sim.submit(_qv(8, s), shots=256, seed=s) for s in range(6)]
    for s, f in enumerate(futs):
        got = f.result(timeout=120).get_counts()
        ref = sim.run(_qv(8, s), shots=256, seed=s, backend="blackwell").get_counts()
        assert got == ref
    from blackwell_backend.hybrid import RoutingPolicy
    assert RoutingPolicy(force_served={"x"}).choose(Circuit(3, name="x")) == "served"


def test_unknown_route_rejected(sim):
    with pytest.raises(ValueError, match="no Aer"):
        sim.run(_qv(4, 1), backend="cuquantum")
    with pytest.raises(ValueError):
        sim.run_statevector(_qv(4, 1, measure=False), backend="served")
    with pytest.raises(ValueError, match="measure"):
        sim.run_statevector(_qv(4, 1), backend="batched")    # collapse needs the plain path


def test_route_summary_prints(sim, capsys):
    sim.print_route_summary()
    out = capsys.readouterr().out
    assert out.startswith("Routing summary:")
    assert "batched" in out and "served" in out
