"""The drop-in surface for Qiskit objects, on the CPU: QuantumCircuit- and
SparsePauliOp-shaped objects (duck-typed, qiskit is not installed here) go
through from_qiskit / PauliSum.from_sparse_pauli_op and the lowering, and the
resulting libqsim op records, run by the FP64 oracle, must equal the circuit
built directly from each instruction's dense matrix.  The reference
transpiles every circuit to its native basis first
(blackwell_backend/simulator.py:489-498); here non-native gates are lowered
by name, by to_matrix(), as controlled gates, or through their definition."""
import cmath
import math

import numpy as np
import pytest
import scipy.linalg as sla

import sv_oracle as O
from qsim_b200 import gates as G
from qsim_b200.circuit import Circuit, from_qiskit, lower
from qsim_b200.paulis import PauliSum


# ------------------------------------------------------- Qiskit-shaped objects
class Bit:
    def __init__(self, i):
        self.i = i


class Op:
    def __init__(self, name, params=(), matrix=None, num_qubits=1, definition=None, base_gate=None,
                 num_ctrl_qubits=0, ctrl_state=None):
        self.name, self.params, self._m = name, list(params), matrix
        self.num_qubits, self.definition = num_qubits, definition
        if base_gate is not None:
            self.base_gate, self.num_ctrl_qubits, self.ctrl_state = base_gate, num_ctrl_qubits, ctrl_state

    def to_matrix(self):
        if self._m is None:
            raise AttributeError("no matrix")
        return self._m


class Inst:
    def __init__(self, op, qubits, clbits=()):
        self.operation, self.qubits, self.clbits = op, tuple(qubits), tuple(clbits)


class QC:
    def __init__(self, n, ncl=0, name="duck"):
        self.qubits = [Bit(i) for i in range(n)]
        self.clbits = [Bit(i) for i in range(ncl)]
        self.num_qubits, self.num_clbits, self.name, self.data = n, ncl, name, []

    def add(self, op, qs, cs=()):
        self.data.append(Inst(op, [self.qubits[q] for q in qs], [self.clbits[c] for c in cs]))
        return self


def _haar(rng, d):
    return G.haar_unitary(rng, d)


def _apply_dense(psi, n, m, qs, controls=()):
    """Reference application of a little-endian matrix on qubits qs."""
    return O._apply_k(psi, n, list(qs), np.asarray(m, dtype=np.complex128), list(controls))


def test_duck_circuit_all_conversion_routes_match_dense():
    rng = np.random.default_rng(1)
    n = 5
    u2 = _haar(rng, 4)          # an "ecr"-like gate known only by its matrix
    u1 = _haar(rng, 2)
    sub = QC(3, name="sub")     # definition of a 3-qubit gate: known gates only
    sub.add(Op("h"), [0]).add(Op("cx"), [0, 2]).add(Op("ry", [0.7]), [1]).add(Op("ccx"), [2, 1, 0])
    qc = QC(n, 1)
    qc.add(Op("h"), [0]).add(Op("cy"), [0, 3]).add(Op("ecr", matrix=u2, num_qubits=2), [4, 1])
    qc.add(Op("my1q", matrix=u1), [2])
    # doubly controlled U on target 4; control 1 must be |0> (ctrl_state 0b10: bit 0 = first control)
    qc.add(Op("c2u", base_gate=Op("u", matrix=u1), num_ctrl_qubits=2, ctrl_state=0b10, num_qubits=3), [1, 3, 4])
    qc.add(Op("my3q", definition=sub, num_qubits=3), [4, 0, 2])
    qc.add(Op("rzz", [0.3]), [1, 2]).add(Op("ecr", matrix=u2, num_qubits=2), [0, 3])
    qc.add(Op("barrier"), []).add(Op("measure"), [0], [0])
    circ = from_qiskit(qc)
    ops = lower(circ)
    got = O.simulate(n, ops)

    psi = O.zero_state(n)
    psi = _apply_dense(psi, n, G.mat1("h"), [0])
    psi = _apply_dense(psi, n, G.mat1("y"), [3], [0])
    psi = _apply_dense(psi, n, u2, [4, 1])
    psi = _apply_dense(psi, n, u1, [2])
    X = G.mat1("x")
    psi = _apply_dense(psi, n, X, [1])
    psi = _apply_dense(psi, n, u1, [4], [1, 3])
    psi = _apply_dense(psi, n, X, [1])
    # definition of my3q on (4, 0, 2): sub-qubits 0 -> 4, 1 -> 0, 2 -> 2
    psi = _apply_dense(psi, n, G.mat1("h"), [4])
    psi = _apply_dense(psi, n, X, [2], [4])
    psi = _apply_dense(psi, n, G.mat1("ry", [0.7]), [0])
    psi = _apply_dense(psi, n, X, [4], [2, 0])
    psi = _apply_dense(psi, n, np.diag(np.diagonal(G.pauli_rot2("z", "z", 0.3))), [1, 2])
    psi = _apply_dense(psi, n, u2, [0, 3])
    assert np.allclose(got, psi, atol=1e-12)
    assert [i.name for i in circ.data][-1] == "measure"


def _pauli(s):
    return {"i": np.eye(2), "x": G._PAULI["x"], "y": G._PAULI["y"], "z": G._PAULI["z"]}[s]


@pytest.mark.parametrize("name,params,nq", [
    ("cy", (), 2), ("ch", (), 2), ("csx", (), 2), ("crx", (0.4,), 2), ("cry", (-1.1,), 2), ("cu1", (0.9,), 2),
    ("cu3", (0.3, 1.2, -0.5), 2), ("cs", (), 2), ("csdg", (), 2), ("ccz", (), 3), ("mcp", (0.6,), 4),
    ("rxx", (0.8,), 2), ("ryy", (-0.4,), 2), ("rzz", (1.3,), 2), ("rzx", (0.25,), 2), ("iswap", (), 2),
    ("dcx", (), 2), ("r", (0.7, -0.2), 1)])
def test_named_gates_against_their_definitions(name, params, nq):
    n = 4
    rng = np.random.default_rng(7)
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi0 /= np.linalg.norm(psi0)
    qs = [2, 0, 3, 1][:nq]
    qc = Circuit(n)
    qc.append(name, qs, params)
    got = O.simulate(n, lower(qc), psi0)
    # independent definitions (Qiskit's documented matrices / exponentials)
    base = {"cy": "y", "ch": "h", "csx": "sx", "crx": "rx", "cry": "ry", "cu3": "u3"}
    phase = {"cu1": cmath.exp(1j * params[0]) if params else 0, "cs": 1j, "csdg": -1j, "ccz": -1.0,
             "mcp": cmath.exp(1j * params[0]) if params else 0}
    if name in base:
        want = _apply_dense(psi0, n, G.mat1(base[name], params), qs[1:], qs[:1])
    elif name in phase:
        want = _apply_dense(psi0, n, np.diag([1, phase[name]]), qs[-1:], qs[:-1])
    elif name in ("rxx", "ryy", "rzz", "rzx"):
        p0, p1 = {"rxx": "xx", "ryy": "yy", "rzz": "zz", "rzx": "zx"}[name]
        M = sla.expm(-0.5j * params[0] * np.kron(_pauli(p1), _pauli(p0)))
        want = _apply_dense(psi0, n, M, qs)
    elif name == "iswap":
        M = sla.expm(0.25j * math.pi * (np.kron(_pauli("x"), _pauli("x")) + np.kron(_pauli("y"), _pauli("y"))))
        want = _apply_dense(psi0, n, M, qs)
    elif name == "dcx":
        X = G.mat1("x")
        want = _apply_dense(_apply_dense(psi0, n, X, [qs[1]], [qs[0]]), n, X, [qs[0]], [qs[1]])
    else:  # r
        th, ph = params
        M = sla.expm(-0.5j * th * (math.cos(ph) * _pauli("x") + math.sin(ph) * _pauli("y")))
        want = _apply_dense(psi0, n, M, qs)
    assert np.allclose(got, want, atol=1e-12), name


def test_unknown_gate_without_matrix_or_definition_is_rejected():
    qc = QC(2).add(Op("mystery", num_qubits=2), [0, 1])
    with pytest.raises(ValueError, match="Unsupported instruction: mystery"):
        from_qiskit(qc)
    qc = QC(1).add(Op("rx", ["theta"]), [0])     # an unbound parameter
    with pytest.raises(ValueError, match="unbound parameter"):
        from_qiskit(qc)


class PauliList:
    def __init__(self, labels):
        n = len(labels[0][1])
        self.x = np.zeros((len(labels), n), dtype=bool)
        self.z = np.zeros((len(labels), n), dtype=bool)
        self.phase = np.zeros(len(labels), dtype=np.int64)
        for k, (ph, lab) in enumerate(labels):
            self.phase[k] = ph
            for pos, ch in enumerate(reversed(lab)):
                self.x[k, pos] = ch in "XY"
                self.z[k, pos] = ch in "YZ"
        # .phase is the label phase, as qiskit's PauliList.phase reports it
        # ("Y" is 0, "-iY" is 1); the internal x/z form's extra i per Y is
        # not part of it


class SPO:
    """SparsePauliOp-shaped: coeffs, paulis (x, z, phase), num_qubits."""

    def __init__(self, labels, coeffs):
        self.paulis = PauliList(labels)
        self.coeffs = np.asarray(coeffs, dtype=np.complex128)
        self.num_qubits = len(labels[0][1])


def test_sparse_pauli_op_duck_with_phases():
    # (-i)^k prefix phases: "-iY" is phase 1, "-Y" phase 2, "iZ" phase 3
    labels = [(0, "XYZ"), (1, "IYI"), (2, "YIY"), (3, "ZIX"), (0, "III")]
    coeffs = [0.5, 1.0 + 0.5j, -0.25, 0.75j, 0.1]
    spo = SPO(labels, coeffs)
    ps = PauliSum.from_sparse_pauli_op(spo)
    want = np.zeros((8, 8), dtype=np.complex128)
    for (ph, lab), c in zip(labels, coeffs):
        M = np.eye(1)
        for ch in lab:
            M = np.kron(M, _pauli(ch.lower()))
        want += c * (-1j) ** ph * M
    np.testing.assert_allclose(ps.to_dense(), want, atol=1e-12)


def test_result_stand_in_has_qiskit_shape():
    from blackwell_backend.simulator import _make_result
    r = _make_result({"0x0": 3, "0x5": 1}, 4, {"name": "c", "n_qubits": 3}, 0.01)
    assert r.get_counts() == {"0x0": 3, "0x5": 1}
    assert r.results[0].header == {"name": "c", "n_qubits": 3}
    assert r.results[0].shots == 4 and r.results[0].success and r.success
    assert r.results[0].data.counts == {"0x0": 3, "0x5": 1}
    assert r.backend_name == "blackwell_simulator" and r.time_taken == 0.01
