"""GPU-resident CSR Hamiltonian (mirrors blackwell_backend/hamiltonian.py:20-79).

``from_sparse_pauli_op`` accepts a qiskit SparsePauliOp (duck-typed) or a
qsim_b200 PauliSum and builds the CSR from the Pauli masks directly in FP64
(the reference goes through qiskit's dense-free to_matrix, hamiltonian.py:58).
"""
from __future__ import annotations

import numpy as np
import torch

from qsim_b200.paulis import PauliSum, csr_from_paulis


class HamiltonianCSR:
    """row_ptr int32 [N+1], col_idx int32 [nnz], values complex64 [nnz] on the
    device; spectral_bound = sum |c| (hamiltonian.py:66)."""

    def __init__(self, row_ptr, col_idx, values, n_qubits, spectral_bound, paulis: PauliSum | None = None):
        self.row_ptr = row_ptr
        self.col_idx = col_idx
        self.values = values
        self.n_qubits = int(n_qubits)
        self.n_rows = 1 << self.n_qubits
        self.nnz = int(col_idx.shape[0])
        self.spectral_bound = float(spectral_bound)
        self.paulis = paulis

    @staticmethod
    def from_sparse_pauli_op(spo, device="cuda") -> "HamiltonianCSR":
        ps = PauliSum.from_sparse_pauli_op(spo)
        rp, ci, val = csr_from_paulis(ps)
        return HamiltonianCSR(torch.from_numpy(rp).to(device), torch.from_numpy(ci).to(device),
                              torch.from_numpy(val).to(device), ps.num_qubits, ps.spectral_bound(), ps)

    from_pauli_sum = from_sparse_pauli_op

    def memory_bytes(self) -> int:
        return int(self.row_ptr.nbytes + self.col_idx.nbytes + self.values.nbytes)

    def __repr__(self):
        return (f"HamiltonianCSR(n_qubits={self.n_qubits}, dim={self.n_rows}, nnz={self.nnz}, "
                f"spectral_bound={self.spectral_bound:.4f}, memory={self.memory_bytes() / 1024:.1f} KB)")
