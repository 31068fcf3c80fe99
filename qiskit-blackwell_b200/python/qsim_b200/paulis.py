"""Pauli sums (a qiskit-free stand-in for SparsePauliOp) and the CSR builder.

A term is (x_mask, z_mask, coef): X on bits of x, Z on bits of z, Y where both
are set, so P = i^{popc(x&z)} X^x Z^z.  Labels follow Qiskit: the rightmost
character acts on qubit 0 (the reference's ab_test.py:376-412 Hamiltonians
are written this way).

``csr_from_paulis`` replaces ``SparsePauliOp.to_matrix(sparse=True).tocsr()``
(blackwell_backend/hamiltonian.py:58): it builds the matrix directly from the
masks in FP64 and rounds the values to complex64 once.
"""
from __future__ import annotations

import numpy as np


class PauliSum:
    def __init__(self, x, z, coefs, num_qubits: int):
        self.x = np.asarray(x, dtype=np.uint64).reshape(-1)
        self.z = np.asarray(z, dtype=np.uint64).reshape(-1)
        self.coefs = np.asarray(coefs, dtype=np.complex128).reshape(-1)
        self.num_qubits = int(num_qubits)
        if not (self.x.size == self.z.size == self.coefs.size):
            raise ValueError("x, z and coefs must have the same length")

    # -- constructors
    @classmethod
    def from_list(cls, terms, num_qubits: int | None = None) -> "PauliSum":
        """terms: iterable of (label, coef), e.g. [("XXI", 0.5), ("IIZ", 1.0)]."""
        xs, zs, cs = [], [], []
        n = num_qubits
        for label, coef in terms:
            label = label.upper()
            if n is None:
                n = len(label)
            if len(label) != n:
                raise ValueError("all labels must have num_qubits characters")
            x = z = 0
            for pos, ch in enumerate(reversed(label)):
                if ch == "X":
                    x |= 1 << pos
                elif ch == "Y":
                    x |= 1 << pos
                    z |= 1 << pos
                elif ch == "Z":
                    z |= 1 << pos
                elif ch != "I":
                    raise ValueError(f"bad Pauli label character {ch!r}")
            xs.append(x)
            zs.append(z)
            cs.append(complex(coef))
        return cls(xs, zs, cs, n or 0)

    @classmethod
    def from_sparse_pauli_op(cls, spo) -> "PauliSum":
        """Duck-typed conversion of qiskit.quantum_info.SparsePauliOp."""
        if isinstance(spo, PauliSum):
            return spo
        paulis = spo.paulis
        X = np.asarray(paulis.x, dtype=bool)
        Z = np.asarray(paulis.z, dtype=bool)
        n = X.shape[1]
        w = (1 << np.arange(n, dtype=np.uint64)).astype(np.uint64)
        x = (X.astype(np.uint64) * w).sum(axis=1).astype(np.uint64)
        z = (Z.astype(np.uint64) * w).sum(axis=1).astype(np.uint64)
        # PauliList.phase is the phase relative to the label (a plain "Y" has
        # phase 0, "-iY" has 1): P = (-i)^phase * label.  Our P is the label
        # product itself (i^{|x&z|} X^x Z^z), so fold (-i)^phase into c.
        phase = np.asarray(getattr(paulis, "phase", np.zeros(len(x))), dtype=np.int64)
        corr = (-1j) ** (phase % 4)
        coefs = np.asarray(spo.coeffs, dtype=np.complex128) * corr
        return cls(x, z, coefs, n)

    # -- properties
    def __len__(self):
        return self.x.size

    def spectral_bound(self) -> float:
        """sum |c| (blackwell_backend/hamiltonian.py:66)."""
        return float(np.sum(np.abs(self.coefs)))

    def real_coefs(self) -> np.ndarray:
        if np.max(np.abs(self.coefs.imag), initial=0.0) > 0:
            raise ValueError("expectation values need real (Hermitian) coefficients")
        return self.coefs.real.astype(np.float64)

    def to_dense(self) -> np.ndarray:
        """FP64 dense matrix (small n only; test/oracle helper)."""
        n = self.num_qubits
        N = 1 << n
        H = np.zeros((N, N), dtype=np.complex128)
        cols = np.arange(N, dtype=np.uint64)
        for x, z, c in zip(self.x, self.z, self.coefs):
            ny = bin(int(x & z)).count("1")
            rows = cols ^ x
            sgn = 1 - 2 * (np.bitwise_count(cols & z) & 1).astype(np.int64)
            H[rows.astype(np.int64), cols.astype(np.int64)] += c * (1j ** ny) * sgn
        return H


def csr_from_paulis(ps: PauliSum, rows_per_chunk: int = 1 << 17):
    """CSR (row_ptr int32, col int32, val complex64) of the Pauli sum, FP64
    accumulation, exact zeros dropped, columns sorted within each row.

    Row r holds one entry per distinct X mask, at column r ^ X.  Rows are
    built in chunks: the entries of a chunk as a [rows, masks] array, each
    row's entries sorted by column, zeros dropped."""
    n = ps.num_qubits
    N = 1 << n
    xs = np.unique(ps.x)
    slot = np.searchsorted(xs, ps.x)
    # FP64 weight of each term: c * i^(number of Y factors)
    w = [c * (1j ** bin(int(x & z)).count("1")) for x, z, c in zip(ps.x, ps.z, ps.coefs)]
    counts = np.zeros(N, dtype=np.int64)
    col_parts, val_parts = [], []
    for r0 in range(0, N, rows_per_chunk):
        rows = np.arange(r0, min(N, r0 + rows_per_chunk), dtype=np.uint64)
        cols_t = xs[:, None] ^ rows[None, :]                             # [nx, R], contiguous per mask
        vals_t = np.zeros(cols_t.shape, dtype=np.complex128)
        for t in range(len(w)):
            k = slot[t]
            sgn = 1.0 - 2.0 * (np.bitwise_count(cols_t[k] & ps.z[t]) & 1)  # sign from column bits & z
            vals_t[k] += w[t] * sgn
        cols, vals = cols_t.T, vals_t.T                                  # [R, nx]
        order = np.argsort(cols, axis=1, kind="stable")
        cols_s = np.take_along_axis(cols, order, axis=1)
        vals_s = np.take_along_axis(vals, order, axis=1)
        keep = vals_s != 0
        counts[r0: r0 + len(rows)] = keep.sum(axis=1)
        col_parts.append(cols_s[keep].astype(np.int32))
        val_parts.append(vals_s[keep].astype(np.complex64))
    row_ptr = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    if row_ptr[-1] >= 2 ** 31:
        raise ValueError("CSR too large for int32 indices")
    return (row_ptr.astype(np.int32), np.concatenate(col_parts) if col_parts else np.zeros(0, np.int32),
            np.concatenate(val_parts) if val_parts else np.zeros(0, np.complex64))
