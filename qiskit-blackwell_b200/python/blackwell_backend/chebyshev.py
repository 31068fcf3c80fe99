"""Chebyshev evolution exp(-iHt)|psi> (mirrors blackwell_backend/chebyshev.py).

Coefficients are computed on the host in FP64 exactly as the reference does
(chebyshev.py:26-78): c_k = (2 - delta_k0) (-i)^k J_k(alpha), alpha =
bound*|t|, degree estimate K = alpha + 2 ln(1/eps) + 20 (at least 10), then the
smallest K whose coefficient tail sum stays below `precision`, K >= 2,
conjugated for t < 0.  The recurrence runs in libqsim: one fused launch per
degree (CSR SpMV + three-term step + accumulation) over three vectors.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch
from scipy.special import jv

from qsim_b200.engine import _h, _ptr, check_state


def chebyshev_coefficients(t, spectral_bound, precision=1e-10):
    """Returns (coeffs complex128 [K+1], K, tail_bound)."""
    alpha = spectral_bound * abs(t)
    k_est = max(int(alpha + 2.0 * np.log(1.0 / precision) + 20), 10)
    coeffs = np.zeros(k_est + 1, dtype=np.complex128)
    for k in range(k_est + 1):
        # Python complex power, as in the reference, so the phases round alike
        coeffs[k] = (2.0 if k > 0 else 1.0) * ((-1j) ** k) * jv(k, alpha)
    cumtail = np.cumsum(np.abs(coeffs)[::-1])[::-1]
    K = k_est
    for kk in range(k_est, 0, -1):
        if cumtail[kk] < precision:
            K = kk
        else:
            break
    K = max(K, 2)
    coeffs = coeffs[: K + 1]
    if t < 0:
        coeffs = np.conj(coeffs)
    tail = float(cumtail[min(K, len(cumtail) - 1)])
    return coeffs, K, tail


def chebyshev_evolve(state, hamiltonian_csr, t, precision=1e-10, bk=None):
    """Returns (result complex64 tensor, info dict with the reference's keys,
    chebyshev.py:160-170)."""
    t0 = time.perf_counter()
    n = check_state(state)
    h = hamiltonian_csr
    if h.n_qubits != n:
        raise RuntimeError("state and Hamiltonian widths differ")
    coeffs, K, tail = chebyshev_coefficients(t, h.spectral_bound, precision)
    scale = 1.0 / h.spectral_bound
    out = torch.empty_like(state)
    work = torch.empty(3 * state.numel(), dtype=torch.complex64, device=state.device)
    cbuf = np.ascontiguousarray(np.stack([coeffs.real, coeffs.imag], axis=-1).reshape(-1), dtype=np.float64)
    _h(state.device.index).call("qs_cheb_evolve", _ptr(h.row_ptr), _ptr(h.col_idx), _ptr(h.values), n, _ptr(state),
                                _ptr(out), cbuf.ctypes.data_as(C.POINTER(C.c_double)), int(K), float(scale),
                                _ptr(work))
    torch.cuda.current_stream(state.device).synchronize()
    elapsed = time.perf_counter() - t0
    info = {
        "engine": "chebyshev-b200",
        "experimental": True,
        "chebyshev_degree": K,
        "spectral_bound": h.spectral_bound,
        "truncation_error_bound": tail,
        "spmv_count": K,
        "workspace_vectors": 3,
        "workspace_bytes": 3 * state.numel() * 8,
        "elapsed_s": elapsed,
    }
    return out, info


def chebyshev_evolve_pauli(state, paulis, t, precision=1e-10):
    """Matrix-free Chebyshev evolution: H given as a Pauli sum (real
    coefficients) is applied on the fly from its X/Z masks; no CSR is built
    or read.  Same coefficients, recurrence and info keys as chebyshev_evolve."""
    t0 = time.perf_counter()
    n = check_state(state)
    if paulis.num_qubits != n:
        raise RuntimeError("state and Hamiltonian widths differ")
    bound = paulis.spectral_bound()
    coeffs, K, tail = chebyshev_coefficients(t, bound, precision)
    x = np.ascontiguousarray(paulis.x, dtype=np.uint64)
    z = np.ascontiguousarray(paulis.z, dtype=np.uint64)
    c = np.ascontiguousarray(paulis.real_coefs(), dtype=np.float64)
    out = torch.empty_like(state)
    work = torch.empty(2 * state.numel(), dtype=torch.complex64, device=state.device)
    cbuf = np.ascontiguousarray(np.stack([coeffs.real, coeffs.imag], axis=-1).reshape(-1), dtype=np.float64)
    _h(state.device.index).call("qs_cheb_evolve_pauli", n, _ptr(state), _ptr(out),
                                x.ctypes.data_as(C.POINTER(C.c_uint64)), z.ctypes.data_as(C.POINTER(C.c_uint64)),
                                c.ctypes.data_as(C.POINTER(C.c_double)), int(len(c)),
                                cbuf.ctypes.data_as(C.POINTER(C.c_double)), int(K), float(1.0 / bound), _ptr(work))
    torch.cuda.current_stream(state.device).synchronize()
    info = {
        "engine": "chebyshev-b200-pauli",
        "experimental": True,
        "chebyshev_degree": K,
        "spectral_bound": bound,
        "truncation_error_bound": tail,
        "spmv_count": K,
        "workspace_vectors": 2,
        "workspace_bytes": 2 * state.numel() * 8,
        "elapsed_s": time.perf_counter() - t0,
    }
    return out, info
