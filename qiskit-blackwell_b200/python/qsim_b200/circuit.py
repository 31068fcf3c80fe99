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
    # Qiskit's other standard gates (lowered to the same op kinds)
    def cy(self, c, t): return self.append("cy", [c, t])
    def ch(self, c, t): return self.append("ch", [c, t])
    def csx(self, c, t): return self.append("csx", [c, t])
    def crx(self, th, c, t): return self.append("crx", [c, t], [th])
    def cry(self, th, c, t): return self.append("cry", [c, t], [th])
    def cu1(self, lam, c, t): return self.append("cu1", [c, t], [lam])
    def cu3(self, th, phi, lam, c, t): return self.append("cu3", [c, t], [th, phi, lam])
    def cs(self, c, t): return self.append("cs", [c, t])
    def csdg(self, c, t): return self.append("csdg", [c, t])
    def ccz(self, a, b, c): return self.append("ccz", [a, b, c])
    def mcp(self, lam, controls, t): return self.append("mcp", list(controls) + [t], [lam])
    def rxx(self, th, a, b): return self.append("rxx", [a, b], [th])
    def ryy(self, th, a, b): return self.append("ryy", [a, b], [th])
    def rzz(self, th, a, b): return self.append("rzz", [a, b], [th])
    def rzx(self, th, a, b): return self.append("rzx", [a, b], [th])
    def iswap(self, a, b): return self.append("iswap", [a, b])
    def dcx(self, a, b): return self.append("dcx", [a, b])
    def r(self, th, phi, q): return self.append("r", [q], [th, phi])

    def mcu(self, matrix, controls, targets):
        """A 2x2 or 4x4 matrix on `targets` (bit 0 = first target), applied
        where every control qubit is |1>."""
        m = np.asarray(matrix, dtype=np.complex128)
        targets = list(targets)
        if len(targets) not in (1, 2) or m.shape != (2 ** len(targets),) * 2:
            raise ValueError("mcu takes a 2x2 matrix on one target or a 4x4 on two")
        return self.append("mcu", list(controls) + targets, [len(targets)], matrix=m)

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


# Instruction names lower() handles directly.
LOWERABLE = (G.NATIVE_1Q | G.NATIVE_2Q | G.NATIVE_MC | set(G.CONTROLLED_1Q) | set(G.CONTROLLED_PHASE)
             | set(G.PAULI_ROT_2Q) | set(NOISE_OPS)
             | {"iswap", "dcx", "r", "unitary", "mcu", "measure", "reset", "barrier"})


def _float_params(op, name):
    out = []
    for p in getattr(op, "params", ()):
        try:
            out.append(float(p))
        except (TypeError, ValueError):
            raise ValueError(f"unbound parameter in {name}") from None
    return out


def _convert(out: Circuit, op, qs, cs, depth: int) -> None:
    """Appends one Qiskit operation acting on qubits `qs` (indices of `out`).

    The reference transpiles every circuit to its native basis before
    compiling it (blackwell_backend/simulator.py:489-498).  Here:
      * gates lower() knows keep their name (and parameters);
      * a controlled gate (num_ctrl_qubits, base_gate, ctrl_state) whose base
        acts on 1 or 2 qubits becomes one multi-controlled op with the base
        gate's matrix; controls that must be |0> are wrapped in exact X gates;
      * any other 1- or 2-qubit gate becomes a `unitary` from to_matrix();
      * anything else is expanded through its `definition` circuit.
    A definition's global phase is dropped, as the reference does (it never
    reads global_phase), so statevectors agree up to a global phase."""
    name = op.name.lower()
    if name == "delay":
        return
    if name == "unitary":
        out.unitary(np.asarray(op.to_matrix()), qs)
        return
    if name in LOWERABLE:
        out.append(name, qs, _float_params(op, name), cs)
        return
    nc = int(getattr(op, "num_ctrl_qubits", 0) or 0)
    base = getattr(op, "base_gate", None)
    if nc > 0 and base is not None and len(qs) - nc in (1, 2) and hasattr(base, "to_matrix"):
        state = getattr(op, "ctrl_state", None)
        state = (1 << nc) - 1 if state is None else (int(state, 2) if isinstance(state, str) else int(state))
        flips = [qs[i] for i in range(nc) if not (state >> i) & 1]
        for q in flips:
            out.x(q)
        if getattr(base, "name", "") == "x" and len(qs) - nc == 1:
            out.mcx(qs[:nc], qs[nc])                  # exact, as the native mcx
        else:
            out.mcu(np.asarray(base.to_matrix()), qs[:nc], qs[nc:])
        for q in flips:
            out.x(q)
        return
    if len(qs) in (1, 2) and hasattr(op, "to_matrix"):
        try:
            m = np.asarray(op.to_matrix(), dtype=np.complex128)
        except Exception:
            m = None
        if m is not None and m.shape == (2 ** len(qs),) * 2:
            out.unitary(m, qs)
            return
    d = getattr(op, "definition", None)
    if d is not None and depth < 32:
        qmap = {q: qs[i] for i, q in enumerate(d.qubits)}
        cmap = {c: cs[i] for i, c in enumerate(getattr(d, "clbits", ())) if i < len(cs)}
        for inst in d.data:
            _convert(out, inst.operation, [qmap[q] for q in inst.qubits], [cmap[c] for c in inst.clbits if c in cmap],
                     depth + 1)
        return
    raise ValueError(f"Unsupported instruction: {name}")


def from_qiskit(qc) -> Circuit:
    """Convert a qiskit.QuantumCircuit (duck-typed: num_qubits, num_clbits,
    qubits, clbits, data of instructions with .operation/.qubits/.clbits)
    into a Circuit; gates outside the lowered set go through _convert."""
    if isinstance(qc, Circuit):
        return qc
    qidx = {q: i for i, q in enumerate(qc.qubits)}
    cidx = {c: i for i, c in enumerate(qc.clbits)}
    out = Circuit(qc.num_qubits, qc.num_clbits, getattr(qc, "name", "circuit"))
    for inst in qc.data:
        _convert(out, inst.operation, [qidx[q] for q in inst.qubits], [cidx[c] for c in inst.clbits], 0)
    return out


# ---------------------------------------------------------------- lowering
def _set_m(rec, mat):
    flat = np.asarray(mat, dtype=np.complex128).reshape(-1)
    rec["m"][: 2 * flat.size: 2] = flat.real
    rec["m"][1: 2 * flat.size: 2] = flat.imag


def lower(circuit: Circuit, strip_measure: bool = True) -> np.ndarray:
    """Circuit -> qs_op structured array (measure/reset/barrier dropped when
    strip_measure, else rejected; they are handled by the backend)."""
    recs = np.zeros(2 * len(circuit.data), dtype=OP_DTYPE)
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
        elif name in G.CONTROLLED_1Q:
            r["kind"] = OP_MCU1
            _set_m(r, G.mat1(G.CONTROLLED_1Q[name], ins.params))
        elif name in G.CONTROLLED_PHASE:
            r["kind"] = OP_MCPHASE
            _set_m(r, [complex(G.CONTROLLED_PHASE[name](ins.params))])
        elif name == "rzz":
            r["kind"] = OP_DIAG2
            _set_m(r, np.diagonal(G.pauli_rot2("z", "z", float(ins.params[0]))))
        elif name in G.PAULI_ROT_2Q:
            r["kind"] = OP_U2
            _set_m(r, G.pauli_rot2(*G.PAULI_ROT_2Q[name], float(ins.params[0])))
        elif name == "iswap":
            r["kind"] = OP_U2
            _set_m(r, G.ISWAP)
        elif name == "r":
            r["kind"] = OP_U1
            _set_m(r, G.r_gate(float(ins.params[0]), float(ins.params[1])))
        elif name == "mcu":
            r["kind"] = OP_MCU1 if int(ins.params[0]) == 1 else OP_MCU2
            _set_m(r, ins.matrix)
        elif name == "dcx":
            # CX(q0 -> q1) then CX(q1 -> q0): two exact permutations
            r["kind"] = OP_MCX
            k += 1
            r2 = recs[k]
            r2["param"], r2["nq"], r2["kind"] = -1, 2, OP_MCX
            r2["q"][:2] = (qs[1], qs[0])
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
