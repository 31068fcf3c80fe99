"""C-ABI state management without torch: allocate, initialise, run a plan,
copy to and from the host, free (the calls a C/C++ host would make)."""
import ctypes as C

import numpy as np
import pytest

import sv_oracle as O
from qsim_b200 import _lib
from qsim_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_state_alloc_run_copy_free():
    L = _lib.load()
    h = _lib.Handle(0)
    n = 14
    st = C.c_void_p()
    h.call("qs_state_alloc", n, C.byref(st))
    assert st.value and st.value % 256 == 0
    try:
        ops = W.qv_ops(n, 6, seed=4)
        h.call("qs_state_init", st, n)
        h.call("qs_run_circuit", st, n, ops.ctypes.data_as(C.POINTER(_lib.QsOp)), len(ops))
        out = np.empty(1 << n, dtype=np.complex64)
        h.call("qs_state_copy_to_host", st, n, out.ctypes.data_as(C.c_void_p))
        assert abs(1 - O.fidelity(out, O.simulate(n, ops))) <= 1e-6
        # round trip through the host
        back = (np.random.default_rng(1).standard_normal(1 << n) + 0j).astype(np.complex64)
        h.call("qs_state_copy_from_host", st, n, back.ctypes.data_as(C.c_void_p))
        out2 = np.empty_like(back)
        h.call("qs_state_copy_to_host", st, n, out2.ctypes.data_as(C.c_void_p))
        assert np.array_equal(back, out2)
    finally:
        h.call("qs_state_free", st)
        h.call("qs_sync")


def test_state_alloc_rejects_bad_width():
    h = _lib.Handle(0)
    st = C.c_void_p()
    with pytest.raises(_lib.QsimError):
        h.call("qs_state_alloc", 0, C.byref(st))
    with pytest.raises(_lib.QsimError):
        h.call("qs_state_alloc", 40, C.byref(st))
