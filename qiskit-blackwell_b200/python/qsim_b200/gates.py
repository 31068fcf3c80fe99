"""FP64 gate matrices (standard Qiskit definitions).

Follows the reference's builders, blackwell_backend/simulator.py:120-242 and
bwk/python/blackwell_kernels/cuquantum.py:133-254,453-498, but in complex128
on the host (the reference builds complex64 tensors on the GPU).  Two-qubit
matrices here use the Qiskit little-endian convention: index bit 0 is the first
listed qubit.  The reference's builders put the first listed qubit in bit 1 and
swap with perm [0,2,1,3] when needed (simulator.py:212-216,290-294).
"""
from __future__ import annotations

import cmath
import math

import numpy as np

I2 = np.eye(2, dtype=np.complex128)
SQ2 = 1.0 / math.sqrt(2.0)


def mat1(name: str, params=()) -> np.ndarray:
    """2x2 matrix of a named single-qubit gate (simulator.py:120-177)."""
    p = [float(x) for x in params]
    if name == "h":
        return np.array([[SQ2, SQ2], [SQ2, -SQ2]], dtype=np.complex128)
    if name == "x":
        return np.array([[0, 1], [1, 0]], dtype=np.complex128)
    if name == "y":
        return np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    if name == "z":
        return np.array([[1, 0], [0, -1]], dtype=np.complex128)
    if name == "s":
        return np.array([[1, 0], [0, 1j]], dtype=np.complex128)
    if name == "sdg":
        return np.array([[1, 0], [0, -1j]], dtype=np.complex128)
    if name == "t":
        return np.array([[1, 0], [0, cmath.exp(1j * math.pi / 4)]], dtype=np.complex128)
    if name == "tdg":
        return np.array([[1, 0], [0, cmath.exp(-1j * math.pi / 4)]], dtype=np.complex128)
    if name == "id":
        return I2.copy()
    if name == "sx":
        return np.array([[0.5 + 0.5j, 0.5 - 0.5j], [0.5 - 0.5j, 0.5 + 0.5j]], dtype=np.complex128)
    if name == "sxdg":
        return np.array([[0.5 - 0.5j, 0.5 + 0.5j], [0.5 + 0.5j, 0.5 - 0.5j]], dtype=np.complex128)
    if name == "rx":
        c, s = math.cos(p[0] / 2), math.sin(p[0] / 2)
        return np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)
    if name == "ry":
        c, s = math.cos(p[0] / 2), math.sin(p[0] / 2)
        return np.array([[c, -s], [s, c]], dtype=np.complex128)
    if name == "rz":
        return np.array([[cmath.exp(-0.5j * p[0]), 0], [0, cmath.exp(0.5j * p[0])]], dtype=np.complex128)
    if name in ("p", "u1"):
        return np.array([[1, 0], [0, cmath.exp(1j * p[0])]], dtype=np.complex128)
    if name == "u2":
        phi, lam = p
        return np.array([[SQ2, -cmath.exp(1j * lam) * SQ2],
                         [cmath.exp(1j * phi) * SQ2, cmath.exp(1j * (phi + lam)) * SQ2]], dtype=np.complex128)
    if name in ("u3", "u"):
        th, phi, lam = p
        c, s = math.cos(th / 2), math.sin(th / 2)
        return np.array([[c, -cmath.exp(1j * lam) * s],
                         [cmath.exp(1j * phi) * s, cmath.exp(1j * (phi + lam)) * c]], dtype=np.complex128)
    raise ValueError(f"Unknown 1Q gate: {name}")


DIAGONAL_1Q = {"z", "s", "sdg", "t", "tdg", "rz", "p", "u1", "id"}
NATIVE_1Q = {"h", "x", "y", "z", "s", "sdg", "t", "tdg", "rx", "ry", "rz", "p", "u1", "u2", "u3", "u", "id", "sx",
             "sxdg"}
NATIVE_2Q = {"cx", "cz", "swap", "cp", "crz", "cu"}
NATIVE_MC = {"ccx", "mcx", "c3x", "c4x", "cswap", "toffoli", "cnot"}

# Qiskit's standard controlled single-qubit gates: name -> the target gate
# (controls first, target last; every control must be |1>).
CONTROLLED_1Q = {"cy": "y", "ch": "h", "csx": "sx", "crx": "rx", "cry": "ry", "cu3": "u3"}
# Controlled phases: name -> function of the params giving the phase applied
# where every listed qubit is |1> (exact as one MCPHASE op).
CONTROLLED_PHASE = {
    "cp": lambda p: cmath.exp(1j * float(p[0])), "cphase": lambda p: cmath.exp(1j * float(p[0])),
    "cu1": lambda p: cmath.exp(1j * float(p[0])), "mcp": lambda p: cmath.exp(1j * float(p[0])),
    "mcphase": lambda p: cmath.exp(1j * float(p[0])), "mcu1": lambda p: cmath.exp(1j * float(p[0])),
    "cs": lambda p: 1j, "csdg": lambda p: -1j, "ccz": lambda p: -1.0,
}
# Two-qubit Pauli rotations exp(-i theta/2 P1 (x) P0), P0 on the first listed
# qubit (Qiskit's RXX/RYY/RZZ/RZX: RZX has Z on the first qubit, X on the second).
PAULI_ROT_2Q = {"rxx": ("x", "x"), "ryy": ("y", "y"), "rzz": ("z", "z"), "rzx": ("z", "x")}
_PAULI = {"x": np.array([[0, 1], [1, 0]], dtype=np.complex128),
          "y": np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
          "z": np.array([[1, 0], [0, -1]], dtype=np.complex128)}


def pauli_rot2(p0: str, p1: str, theta: float) -> np.ndarray:
    """exp(-i theta/2 P1 (x) P0) as a 4x4 with index bit 0 = the qubit of P0."""
    P = np.kron(_PAULI[p1], _PAULI[p0])
    return math.cos(theta / 2) * np.eye(4, dtype=np.complex128) - 1j * math.sin(theta / 2) * P


def r_gate(theta: float, phi: float) -> np.ndarray:
    """Qiskit's RGate: exp(-i theta/2 (cos(phi) X + sin(phi) Y))."""
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return np.array([[c, -1j * cmath.exp(-1j * phi) * s], [-1j * cmath.exp(1j * phi) * s, c]], dtype=np.complex128)


ISWAP = np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)


def cu_target(params) -> np.ndarray:
    """Target block of cu(theta, phi, lam, gamma) (simulator.py:199-208)."""
    th, phi, lam, gam = [float(x) for x in params]
    return cmath.exp(1j * gam) * mat1("u", (th, phi, lam))


def mat2_little(name: str, params=()) -> np.ndarray:
    """4x4 of a named two-qubit gate with bit 0 = first listed qubit
    (the control for cx/cp/crz/cu)."""
    if name == "cx":
        m = np.eye(4, dtype=np.complex128)
        m[[1, 3]] = m[[3, 1]]
        return m
    if name == "cz":
        return np.diag([1, 1, 1, -1]).astype(np.complex128)
    if name == "swap":
        return np.eye(4, dtype=np.complex128)[[0, 2, 1, 3]]
    if name == "cp":
        return np.diag([1, 1, 1, cmath.exp(1j * float(params[0]))]).astype(np.complex128)
    if name == "crz":
        th = float(params[0])
        return np.diag([1, cmath.exp(-0.5j * th), 1, cmath.exp(0.5j * th)]).astype(np.complex128)
    if name == "cu":
        u = cu_target(params)
        m = np.eye(4, dtype=np.complex128)
        # control = bit 0 set: indices 1 (target 0) and 3 (target 1)
        m[1, 1], m[1, 3], m[3, 1], m[3, 3] = u[0, 0], u[0, 1], u[1, 0], u[1, 1]
        return m
    raise ValueError(f"Unknown 2Q gate: {name}")


def haar_unitary(rng: np.random.Generator, dim: int, count: int | None = None) -> np.ndarray:
    """Haar-random U(dim): QR of (G1 + i G2)/sqrt(2) with R's diagonal phases
    moved into Q (the method of bwk/python/blackwell_kernels/qv8.py:55-73)."""
    shape = (dim, dim) if count is None else (count, dim, dim)
    z = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=-2, axis2=-1)
    ph = d / np.abs(d)
    return q * ph[..., np.newaxis, :]
