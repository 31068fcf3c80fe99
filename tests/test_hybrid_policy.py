"""Host-side routing: analyze_circuit counts and RoutingPolicy decisions
(reference blackwell_backend/hybrid.py:51-138), and the seeded uniforms the
routes share with the serving runtime."""
import numpy as np

from blackwell_backend.hybrid import RoutingPolicy, analyze_circuit
from qsim_b200.circuit import Circuit
from qsim_b200.engine import seed_uniforms


def _mixed():
    qc = Circuit(3, 3, name="mixed")
    qc.h(0)
    qc.cx(0, 1)
    qc.barrier()
    qc.unitary(np.eye(4), [1, 2])
    qc.ccx(0, 1, 2)
    qc.measure(2, 2)
    return qc


def _qv_like(n, name="qv"):
    rng = np.random.default_rng(1)
    qc = Circuit(n, name=name)
    for a in range(0, n - 1, 2):
        m, _ = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))
        qc.unitary(m, [a, a + 1])
    qc.h(0)
    return qc


def test_analyze_counts_like_reference():
    a = analyze_circuit(_mixed())
    # barrier skipped; unitary is the only name outside the reference's table
    assert a["num_qubits"] == 3
    assert a["total_gates"] == 5
    assert a["native_gates"] == 4 and a["non_native_gates"] == 1
    assert a["non_native_ratio"] == 0.2
    assert (a["n_1q"], a["n_2q"], a["n_mcx"]) == (2, 2, 1)
    assert a["gate_names"] == {"h", "cx", "unitary", "ccx", "measure"}


def test_analyze_empty_circuit():
    a = analyze_circuit(Circuit(2))
    assert a["total_gates"] == 0 and a["non_native_ratio"] == 0.0


def test_policy_single_and_lists():
    p = RoutingPolicy()
    qc = _mixed()
    assert p.choose(qc) == "blackwell"
    assert p.choose(qc, batch_size=4) == "batched"
    wide = Circuit(24, name="wide")
    wide.h(0)
    assert p.choose(wide, batch_size=4) == "blackwell"      # wider than batch_max_qubits


def test_policy_non_native_threshold():
    p = RoutingPolicy(batch_min_circuits=8)
    native = Circuit(6, name="native")
    native.h(0)
    assert p.choose(native, batch_size=2) == "blackwell"    # short list, native gates
    assert p.choose(_qv_like(6), batch_size=2) == "batched"  # unitary-dense
    assert p.choose(_qv_like(6)) == "blackwell"              # alone
    assert RoutingPolicy(non_native_threshold=1.0, batch_min_circuits=8).choose(_qv_like(6), batch_size=2) \
        == "blackwell"


def test_policy_forced_names():
    p = RoutingPolicy(force_blackwell={"a"}, force_cuquantum={"b"}, force_batched={"c"}, force_served={"d"})
    assert p.choose(_qv_like(4, "a"), batch_size=10) == "blackwell"
    assert p.choose(_qv_like(4, "b")) == "batched"
    assert p.choose(_qv_like(4, "c")) == "batched"
    assert p.choose(_qv_like(4, "d")) == "served"


def test_seed_uniforms_match_splitmix_loop():
    def loop(seed, count):
        m = 2 ** 64 - 1
        x, out = seed, []
        for _ in range(count):
            x = (x + 0x9E3779B97F4A7C15) & m
            z = x
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
            z ^= z >> 31
            out.append((z >> 11) * 2.0 ** -53)
        return np.array(out)
    for s in (0, 7, 2 ** 63 + 5, 2 ** 64 - 1):
        u = seed_uniforms(s, 257)
        assert np.array_equal(u, loop(s, 257))
        assert u.min() >= 0.0 and u.max() < 1.0
    assert seed_uniforms(3, 0).shape == (0,)


def test_policy_keeps_noisy_circuits_on_plain_path():
    qc = Circuit(4, name="noisy")
    qc.h(0)
    qc.amplitude_damp(0.1, 0)
    p = RoutingPolicy()
    assert p.choose(qc, batch_size=8) == "blackwell"
