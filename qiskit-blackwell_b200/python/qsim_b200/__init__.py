"""qsim_b200 — host runtime of the B200 statevector engine.

* ``_lib``      ctypes binding of libqsim.so (C ABI: include/qsim.h)
* ``circuit``   qiskit-free circuit IR and its lowering to libqsim ops
* ``gates``     FP64 gate matrices
* ``paulis``    Pauli sums and the CSR builder
* ``engine``    torch-facing calls (plans, batch plans, reductions, adjoint)
* ``workloads`` seeded synthetic circuits, observables and Hamiltonians
"""
from .circuit import Circuit, OP_DTYPE, from_qiskit, lower  # noqa: F401
from .paulis import PauliSum, csr_from_paulis  # noqa: F401

__version__ = "0.1.0"
