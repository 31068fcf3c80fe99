"""Qiskit-free circuit IR and its lowering to the libqsim op array.

``Circuit`` mirrors the subset of ``qiskit.QuantumCircuit`` that the
reference backend accepts (blackwell_backend/simulator.py:100-109,261-306):
the native 1Q set, cx/cz/swap/cp/crz/cu, ccx/mcx, cswap, measure, reset and
barrier, plus ``unitary`` for arbitrary 1Q/2Q matrices.  ``from_qiskit``
converts a real QuantumCircuit when qiskit is installed.

``lower`` produces a numpy structured array with the exact layout of
``qs_op`` (include/qsim.h), so it can be handed to the C ABI without copies.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import gates as G
from ._lib import (OP_DIAG1, OP_MCPHASE, OP_MCSWAP, OP_MCU1, OP_MCX, OP_RX, OP_RY, OP_RZ, OP_U1, OP_U2, OP_Y,
                   OP_MCU2, OP_DIAG2, OP_AMP_DAMP, OP_DEPHASE, OP_DEPOLARIZE)

# Stochastic channels (one qubit, one probability parameter); only the
# noise-trajectory runner accepts them.
NOISE_OPS = {"depolarize": OP_DEPOLARIZE, "amplitude_damp": OP_AMP_DAMP, "dephase": OP_DEPHASE}

OP_DTYPE = np.dtype([("kind", "<i4"), ("nq", "<i4"), ("q", "<i4", (8,)), ("param", "<i4"), ("flags", "<i4"),
                     ("m", "<f8", (32,))])
assert OP_DTYPE.itemsize == 304


@dataclass
class Instruction:
    name: str
    qubits: tuple
    params: tuple = ()
    clbits: tuple = ()
    matrix: np.ndarray | None = None
    param_index: int = -1   # for trainable rotations (adjoint)


@dataclass
class Circuit:
    num_qubits: int
    num_clbits: int = 0
    name: str = "circuit"
    data: list = field(default_factory=list)

    # -- generic
    def append(self, name, qubits, params=(), clbits=(), matrix=None, param_index=-1):
        qubits = tuple(int(q) for q in qubits)
        for q in qubits:
            if not 0 <= q < self.num_qubits:
                raise ValueError(f"qubit {q} out of range for a {self.num_qubits}-qubit circuit")
        if len(set(qubits)) != len(qubits):
            raise ValueError(f"repeated qubit in {name}{qubits}")
        self.data.append(Instruction(name, qubits, tuple(params), tuple(clbits), matrix, param_index))
        return self

    # -- 1Q (Qiskit argument order: params first, then qubits)
    def h(self, q): return self.append("h", [q])
    def x(self, q): return self.append("x", [q])
    def y(self, q): return self.append("y", [q])
    def z(self, q): return self.append("z", [q])
    def s(self, q): return self.append("s", [q])
    def sdg(self, q): return self.append("sdg", [q])
    def t(self, q): return self.append("t", [q])
    def tdg(self, q): return self.append("tdg", [q])
    def sx(self, q): return self.append("sx", [q])
    def sxdg(self, q): return self.append("sxdg", [q])
    def id(self, q): return self.append("id", [q])
    def rx(self, th, q, param_index=-1): return self.append("rx", [q], [th], param_index=param_index)
    def ry(self, th, q, param_index=-1): return self.append("ry", [q], [th], param_index=param_index)
    def rz(self, th, q, param_index=-1): return self.append("rz", [q], [th], param_index=param_index)
    def p(self, lam, q): return self.append("p", [q], [lam])
    def u1(self, lam, q): return self.append("u1", [q], [lam])
    def u2(self, phi, lam, q): return self.append("u2", [q], [phi, lam])
    def u3(self, th, phi, lam, q): return self.append("u3", [q], [th, phi, lam])
    def u(self, th, phi, lam, q): return self.append("u", [q], [th, phi, lam])

    # -- 2Q / multi-qubit
    def cx(self, c, t): return self.append("cx", [c, t])
    cnot = cx
    def cz(self, a, b): return self.append("cz", [a, b])
    def swap(self, a, b): return self.append("swap", [a, b])
    def cp(self, lam, c, t): return self.append("cp", [c, t], [lam])
    def crz(self, th, c, t): return self.append("crz", [c, t], [th])
    def cu(self, th, phi, lam, gam, c, t): return self.append("cu", [c, t], [th, phi, lam, gam])
    def ccx(self, c1, c2, t): return self.append("ccx", [c1, c2, t])
    toffoli = ccx
    def mcx(self, controls, t): return self.append("mcx", list(controls) + [t])
    def cswap(self, c, a, b): return self.append("cswap", [c, a, b])
    def unitary(self, matrix, qubits):
        m = np.asarray(matrix, dtype=np.complex128)
        qubits = list(qubits)
        if m.shape != (2 ** len(qubits),) * 2 or len(qubits) not in (1, 2):
            raise ValueError("unitary supports 1- and 2-qubit matrices")
        return self.append("unitary", qubits, matrix=m)

    # -- noise channels (noise_sm120.cu semantics; run by qsim_b200.noise)
    def depolarize(self, p, q): return self.append("depolarize", [q], [p])
    def amplitude_damp(self, gamma, q): return self.append("amplitude_damp", [q], [gamma])
    def dephase(self, lam, q): return self.append("dephase", [q], [lam])

    # -- non-unitary
    def measure(self, q, c): return self.append("measure", [q], clbits=[c])
    def reset(self, q): return self.append("reset", [q])
    def barrier(self, *qs): return self.append("barrier", [])

    def copy(self):
        return Circuit(self.num_qubits, self.num_clbits, self.name, list(self.data))

    def size(self):
        return sum(1 for i in self.data if i.name not in ("barrier",))


def from_qiskit(qc) -> Circuit:
    """Convert a qiskit.QuantumCircuit (duck-typed) into a Circuit."""
    if isinstance(qc, Circuit):
        return qc
    qidx = {q: i for i, q in enumerate(qc.qubits)}
    cidx = {c: i for i, c in enumerate(qc.clbits)}
    out = Circuit(qc.num_qubits, qc.num_clbits, getattr(qc, "name", "circuit"))
    for inst in qc.data:
        op = inst.operation
        name = op.name.lower()
        qs = [qidx[q] for q in inst.qubits]
        cs = [cidx[c] for c in inst.clbits]
        params = []
        for p in op.params:
            try:
                params.append(float(p))
            except (TypeError, ValueError):
                if name == "unitary":
                    continue
                raise ValueError(f"unbound parameter in {name}")
        if name == "unitary":
            out.unitary(np.asarray(op.to_matrix()), qs)
        else:
            out.append(name, qs, params, cs)
    return out


# ---------------------------------------------------------------- lowering
def _set_m(rec, mat):
    flat = np.asarray(mat, dtype=np.complex128).reshape(-1)
    rec["m"][: 2 * flat.size: 2] = flat.real
    rec["m"][1: 2 * flat.size: 2] = flat.imag


def lower(circuit: Circuit, strip_measure: bool = True) -> np.ndarray:
    """Circuit -> qs_op structured array (measure/reset/barrier dropped when
    strip_measure, else rejected; they are handled by the backend)."""
    recs = np.zeros(len(circuit.data), dtype=OP_DTYPE)
    k = 0
    for ins in circuit.data:
        name, qs = ins.name, ins.qubits
        if name == "barrier":
            continue
        if name in ("measure", "reset"):
            if strip_measure:
                continue
            raise ValueError("measure/reset cannot be lowered to a unitary program")
        r = recs[k]
        r["param"] = -1
        r["nq"] = len(qs)
        r["q"][: len(qs)] = qs
        if name in ("rx", "ry", "rz") and ins.param_index >= 0:
            r["kind"] = {"rx": OP_RX, "ry": OP_RY, "rz": OP_RZ}[name]
            r["m"][0] = float(ins.params[0])
            r["param"] = ins.param_index
        elif name == "unitary":
            r["kind"] = OP_U1 if len(qs) == 1 else OP_U2
            _set_m(r, ins.matrix)
        elif name in NOISE_OPS:
            r["kind"] = NOISE_OPS[name]
            r["m"][0] = float(ins.params[0])
        elif name == "y":
            r["kind"] = OP_Y
        elif name in G.DIAGONAL_1Q:
            r["kind"] = OP_DIAG1
            m = G.mat1(name, ins.params)
            _set_m(r, [m[0, 0], m[1, 1]])
        elif name in G.NATIVE_1Q:
            r["kind"] = OP_U1
            _set_m(r, G.mat1(name, ins.params))
        elif name in ("cx", "cnot", "ccx", "toffoli", "mcx", "c3x", "c4x"):
            r["kind"] = OP_MCX
        elif name == "cz":
            r["kind"] = OP_MCPHASE
            _set_m(r, [-1.0])
        elif name == "cp":
            r["kind"] = OP_MCPHASE
            _set_m(r, [complex(math.cos(ins.params[0]), math.sin(ins.params[0]))])
        elif name == "swap":
            r["kind"] = OP_MCSWAP
        elif name == "cswap":
            r["kind"] = OP_MCSWAP
        elif name == "crz":
            r["kind"] = OP_MCU1
            _set_m(r, G.mat1("rz", ins.params))
        elif name == "cu":
            r["kind"] = OP_MCU1
            _set_m(r, G.cu_target(ins.params))
        else:
            raise ValueError(f"Unsupported instruction: {name}")
        k += 1
    return recs[:k]


def op_u2(q0: int, q1: int, m4: np.ndarray) -> np.ndarray:
    r = np.zeros(1, dtype=OP_DTYPE)
    r["kind"], r["nq"], r["param"] = OP_U2, 2, -1
    r["q"][0, :2] = (q0, q1)
    _set_m(r[0], m4)
    return r
