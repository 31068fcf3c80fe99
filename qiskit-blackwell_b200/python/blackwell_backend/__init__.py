"""Qiskit backend on the B200 statevector engine (libqsim.so, sm_100a).

Mirrors the reference's blackwell_backend/__init__.py:11-13 exports for the
hot path (BlackwellSimulator) and HybridSimulator (routing among the plain,
batched and served paths); HamiltonianCSR and the Chebyshev driver are
re-exported for run_hamiltonian users.
"""
from .simulator import BlackwellSimulator, Result, counts_from_samples  # noqa: F401
from .hamiltonian import HamiltonianCSR  # noqa: F401
from .chebyshev import chebyshev_coefficients, chebyshev_evolve, chebyshev_evolve_pauli  # noqa: F401
from .hybrid import HybridSimulator, RoutingPolicy, analyze_circuit  # noqa: F401
from .backend import BlackwellBackend  # noqa: F401

__all__ = ["BlackwellSimulator", "HamiltonianCSR", "chebyshev_coefficients", "chebyshev_evolve", "Result",
           "HybridSimulator", "RoutingPolicy", "analyze_circuit", "BlackwellBackend"]
