"""The backend surface on the GPU: run_and_time, CircuitGraph replay, the
device counts histogram (qs_counts), the BackendV2-shaped backend, and
Qiskit-shaped circuits with non-native gates through run_statevector."""
import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200 import engine as E
from qsim_b200 import gates as G
from qsim_b200 import workloads as W
from qsim_b200.circuit import Circuit, from_qiskit, lower

pytestmark = pytest.mark.gpu


def _ghz(n):
    qc = Circuit(n, name=f"ghz{n}")
    qc.h(0)
    for q in range(1, n):
        qc.cx(q - 1, q)
    return qc


def test_run_and_time_shape_and_counts():
    """simulator.py:615-657: warm-up runs, timed repeats, then a final run;
    (Result, {times_s, median_s, min_s, mean_s})."""
    from blackwell_backend import BlackwellSimulator
    sim = BlackwellSimulator()
    qc = Circuit(10, name="qv10")
    for r in W.qv_ops(10, 10, 3):
        m = np.array(r["m"][0:32:2] + 1j * r["m"][1:32:2]).reshape(4, 4)
        qc.unitary(m, [int(r["q"][0]), int(r["q"][1])])
    res, st = sim.run_and_time(qc, shots=1000, seed=5, warmup=1, repeats=3)
    assert set(st) == {"times_s", "median_s", "min_s", "mean_s"} and len(st["times_s"]) == 3
    assert 0 < st["min_s"] <= st["median_s"] <= max(st["times_s"])
    counts = res.get_counts()
    assert sum(counts.values()) == 1000 and res.results[0].header == {"name": "qv10", "n_qubits": 10}
    assert counts == sim.run(qc, shots=1000, seed=5).get_counts()     # same seed, same shots


def test_circuit_graph_replay_matches_oracle():
    """cuquantum.py:101-130: the constructor applies the gates once (warm-up)
    and captures them; each replay applies them again on the same state."""
    import blackwell_kernels as bk
    n = 12
    rng = np.random.default_rng(4)
    mats = [G.haar_unitary(rng, 2) for _ in range(9)]
    targets = [0, 5, 11, 3, 3, 7, 1, 10, 6]
    gates = torch.tensor(np.stack(mats).astype(np.complex64), device="cuda")
    state = bk.state_init(n)
    cg = bk.CircuitGraph(state, gates, targets)
    cg.replay()
    cg.replay()
    torch.cuda.synchronize()
    ops = []
    for _ in range(3):
        c = Circuit(n)
        for m, t in zip(mats, targets):
            c.unitary(m.astype(np.complex64).astype(np.complex128), [t])
        ops.append(lower(c))
    ref = O.simulate(n, np.concatenate(ops))
    got = state.cpu().numpy()
    assert abs(1 - O.fidelity(got, ref)) <= 1e-6 and O.max_abs_err(got, ref) < 1e-5


@pytest.mark.parametrize("n_shots,hi", [(1, 4), (1000, 8), (200_000, 1 << 20), (70_000, 1 << 34)])
def test_counts_histogram_equals_numpy(n_shots, hi):
    rng = np.random.default_rng(n_shots)
    shots = rng.integers(0, hi, size=n_shots, dtype=np.int64)
    got = E.counts(torch.from_numpy(shots).cuda())
    vals, cnt = np.unique(shots, return_counts=True)
    assert list(got.items()) == [(int(v), int(c)) for v, c in zip(vals, cnt)]
    assert E.counts(torch.zeros(0, dtype=torch.int64, device="cuda")) == {}


def test_backend_v2_shape_runs_lists_and_options():
    from blackwell_backend import BlackwellBackend, BlackwellSimulator
    be = BlackwellBackend(shots=512)
    try:
        assert "cx" in be.target and "rzz" in be.target and be.target.instruction_supported("h", (0,))
        assert not be.target.instruction_supported("h", (40,)) and be.max_circuits is None
        assert be.options.shots == 512
        circs = [_ghz(5), _ghz(9), _ghz(3)]
        job = be.run(circs, shots=2000, seed_simulator=11)
        res = job.result()
        assert job.done() and job.status() == "DONE" and job.job_id().startswith("blackwell-")
        assert len(res.results) == 3 and res.success
        for k, n in enumerate((5, 9, 3)):
            c = res.get_counts(k)
            assert set(c) <= {hex(0), hex((1 << n) - 1)} and sum(c.values()) == 2000
            assert res.results[k].header == {"name": f"ghz{n}", "n_qubits": n}
        one = be.run(_ghz(4)).result()
        assert sum(one.get_counts().values()) == 512
        be.set_options(shots=100)
        assert sum(be.run(_ghz(4)).result().get_counts().values()) == 100
        with pytest.raises(AttributeError):
            be.set_options(noise_model=None)
    finally:
        be.close()
    assert BlackwellSimulator is not None


def test_qiskit_shaped_non_native_gates_on_the_gpu():
    """A QuantumCircuit-shaped object with gates outside the native set
    (known names, a matrix-only 2Q gate, a controlled gate with a |0>
    control, a gate known only by its definition) runs on the plan path and
    matches the FP64 oracle run of its lowering."""
    from blackwell_backend import BlackwellSimulator
    from test_qiskit_frontend import QC, Op
    rng = np.random.default_rng(2)
    u2, u1 = G.haar_unitary(rng, 4), G.haar_unitary(rng, 2)
    sub = QC(2, name="sub").add(Op("ch"), [0, 1]).add(Op("rzx", [0.4]), [1, 0])
    n = 14
    qc = QC(n, name="duck")
    for q in range(n):
        qc.add(Op("ry", [0.1 + 0.2 * q]), [q])
    qc.add(Op("ecr", matrix=u2, num_qubits=2), [13, 2]).add(Op("cy"), [4, 9]).add(Op("iswap"), [0, 12])
    qc.add(Op("c2u", base_gate=Op("u", matrix=u1), num_ctrl_qubits=2, ctrl_state=0b01, num_qubits=3), [1, 7, 11])
    qc.add(Op("blk", definition=sub, num_qubits=2), [6, 3]).add(Op("rxx", [0.9]), [5, 8]).add(Op("dcx"), [10, 2])
    qc.add(Op("mcx_gray", base_gate=Op("x", matrix=G.mat1("x")), num_ctrl_qubits=3, num_qubits=4), [0, 1, 2, 13])
    sv, _ = BlackwellSimulator().run_statevector(qc)
    ref = O.simulate(n, lower(from_qiskit(qc)))
    assert abs(1 - O.fidelity(sv, ref)) <= 1e-6 and O.max_abs_err(sv, ref) < 1e-5
