"""blackwell_kernels — drop-in replacement of the reference's Python kernel API
(bwk/python/blackwell_kernels/cuquantum.py, __init__.py:11-33) on top of
libqsim.so (sm_100a).  Same function names, argument meaning and in-place
semantics; every call runs on torch's current CUDA stream.  There is no CPU
path: without the library or a GPU the calls raise.
"""
from .cuquantum import (  # noqa: F401
    apply_gate, apply_gate_2q, apply_gates_fused, apply_gates_reg_tiled,
    apply_diagonal, apply_diagonal_phase, apply_diagonal_2q, state_init,
    measure_qubit, measure_probs, sample,
    expectation_z, expectation_pauli,
    apply_mcgate, apply_mc2qgate, swap_gate, cswap_gate, pauli_x_gate,
    apply_gate_batched, apply_gates_batched_fused, state_init_batched,
    CircuitGraph, hadamard_gate, random_unitary,
    cnot_gate, cz_gate, random_unitary_4x4,
    rz_gate_diag, phase_gate_diag, t_gate_diag, s_gate_diag, z_gate_diag, cz_gate_diag,
    renormalize,
    spmv_csr, chebyshev_step, chebyshev_accum, chebyshev_step_accum,
    apply_depolarizing, apply_amplitude_damping, apply_dephasing,
)
from .qv import (  # noqa: F401
    qv8_simulate, qv4_simulate_cuda, generate_qv8_circuits, heavy_output_probability,
)

__version__ = "0.1.0"
