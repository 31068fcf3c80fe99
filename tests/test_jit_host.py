"""Pass specialisation, host side (no GPU): every tile pass of a plan is
turned into CUDA source and compiled for sm_100a with NVRTC.  Covers every
device-op kind (dense 1Q/2Q, rotations, Kronecker layers, exact X/Y/SWAP,
merged diagonal tables with group, sign and cross terms, controls on tile and
on global qubits) at several tile and register-block widths."""
import ctypes as C

import numpy as np
import pytest

import __graft_entry__  # noqa: F401  (puts the package on sys.path)
from qsim_b200 import _lib
from qsim_b200 import workloads as W
from test_oracle_golden import _random_ops


@pytest.fixture(scope="module")
def L():
    import os
    if not os.path.exists(_lib.lib_path()):
        __graft_entry__.build()
    return _lib.load()


def jit_check(L, n, ops, tile_bits=0, block_bits=0):
    ops = np.ascontiguousarray(ops)
    npass = C.c_int(0)
    rc = L.qs_plan_jit_check(n, ops.ctypes.data_as(C.POINTER(_lib.QsOp)), len(ops), tile_bits, block_bits,
                             C.byref(npass))
    if rc != 0:
        msg = (L.qs_last_error(None) or b"").decode()
        if "libnvrtc" in msg:
            pytest.skip(msg)
        raise AssertionError(msg[:2000])
    return npass.value


@pytest.mark.parametrize("n,tile_bits,block_bits", [(6, 10, 5), (13, 10, 4), (15, 12, 3), (17, 13, 5), (17, 10, 2),
                                                    (16, 12, 6)])
def test_random_all_kinds_compile(L, n, tile_bits, block_bits):
    rng = np.random.default_rng(4000 + n)
    ops = _random_ops(n, 80, rng)
    assert jit_check(L, n, ops, tile_bits, block_bits) >= 1


def test_qv_compiles(L):
    assert jit_check(L, 12, W.qv_ops(12, 12, 0), 10) == 1


def test_layers_with_toffoli_compiles(L):
    assert jit_check(L, 20, W.layers_ops(20, 5, seed=2), 13, 4) >= 2
