"""The allocation-free expectation entry point, called through the C ABI.

qs_expect_pauli_sum_noalloc exists for callers that cannot let a library
allocate device or pinned memory behind their back (a runtime that owns all
of HBM through its own arena and budget, or a latency-critical loop that must
not pay cudaMalloc/cudaFree's implicit synchronisation).  Its scratch is a
fixed static device array shared by all calls, so this test checks two calls
in a row against the allocating entry point, qs_expect_pauli_sum.  It lives
in its own file, collected last, and needs nothing from the other tests.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _observable(n, n_terms, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros(n_terms, dtype=np.uint64)
    z = np.zeros(n_terms, dtype=np.uint64)
    for k in range(n_terms):
        for q in rng.choice(n, min(n, int(rng.integers(1, 5))), replace=False):
            p = int(rng.integers(1, 4))          # 1 = X, 2 = Y, 3 = Z
            if p in (1, 2):
                x[k] |= np.uint64(1 << int(q))
            if p in (2, 3):
                z[k] |= np.uint64(1 << int(q))
    c = rng.standard_normal(n_terms)
    return x, z, np.ascontiguousarray(c, dtype=np.float64)


def _state(n, seed):
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    return torch.from_numpy(psi.astype(np.complex64)).cuda()


def test_noalloc_expectation_matches_allocating_entry_point():
    from qsim_b200 import _lib
    L = _lib.load()
    h = C.c_void_p()
    assert L.qs_create(0, C.byref(h)) == 0
    try:
        u64 = C.POINTER(C.c_uint64)
        f64 = C.POINTER(C.c_double)
        # two calls in a row, then the two ends of the fixed scratch: the
        # full 1024-term table with all 1024 block partials (n = 22), and a
        # one-qubit state (one block)
        for call, (n, nt) in enumerate([(14, 200), (18, 64), (22, 1024), (1, 3)]):
            s = _state(n, 10 + call)
            x, z, c = _observable(n, nt, 20 + call)
            torch.cuda.synchronize()
            ref, got = C.c_double(), C.c_double()
            assert L.qs_expect_pauli_sum(h, C.c_void_p(s.data_ptr()), n, x.ctypes.data_as(u64),
                                         z.ctypes.data_as(u64), c.ctypes.data_as(f64), nt, C.byref(ref)) == 0, \
                L.qs_last_error(h)
            assert L.qs_expect_pauli_sum_noalloc(h, C.c_void_p(s.data_ptr()), n, x.ctypes.data_as(u64),
                                                 z.ctypes.data_as(u64), c.ctypes.data_as(f64), nt,
                                                 C.byref(got)) == 0, L.qs_last_error(h)
            # same slicing and summation order as the allocating entry point
            assert abs(got.value - ref.value) <= 1e-12 * max(1.0, abs(ref.value))
        # sizes beyond the static scratch are rejected with a clear error
        x, z, c = _observable(10, 1025, 3)
        s = _state(10, 4)
        rc = L.qs_expect_pauli_sum_noalloc(h, C.c_void_p(s.data_ptr()), 10, x.ctypes.data_as(u64),
                                           z.ctypes.data_as(u64), c.ctypes.data_as(f64), 1025, C.byref(C.c_double()))
        assert rc == _lib.QS_ERR_INVALID and b"1024" in L.qs_last_error(h)
    finally:
        L.qs_destroy(h)
