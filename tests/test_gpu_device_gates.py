"""Gates given as CUDA tensors: blackwell_kernels passes their device
pointers (qs_apply_*_dev), so no host copy or stream synchronisation happens
per call.  Results must be bit-identical to the host-matrix entry points."""
import ctypes as C

import numpy as np
import pytest
import torch

import blackwell_kernels as bk
from qsim_b200 import _lib
from qsim_b200 import engine as E

pytestmark = pytest.mark.gpu


def _state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return torch.from_numpy((v / np.linalg.norm(v)).astype(np.complex64)).cuda()


def _bits(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("t", [0, 1, 6])
def test_1q_and_diag_device_equals_host(t):
    g = bk.random_unitary().contiguous()          # CUDA complex64 [2, 2]
    d = bk.rz_gate_diag(0.37)
    a, b = _state(9, 1), _state(9, 1)
    bk.apply_gate(a, g, t)
    bk.apply_gate(b, g.cpu(), t)                  # host path
    assert np.array_equal(_bits(a), _bits(b))
    bk.apply_diagonal(a, d, t)
    bk.apply_diagonal(b, d.cpu(), t)
    assert np.array_equal(_bits(a), _bits(b))


@pytest.mark.parametrize("q0,q1", [(0, 5), (3, 8), (7, 2)])
def test_2q_device_equals_host(q0, q1):
    g = bk.random_unitary_4x4().contiguous()
    a, b = _state(9, 2), _state(9, 2)
    bk.apply_gate_2q(a, g, q0, q1)
    bk.apply_gate_2q(b, g.cpu(), q0, q1)
    assert np.array_equal(_bits(a), _bits(b))
    # the C ABI with q0 > q1 (index bit 0 on q0): the kernel swaps bits on load
    h = E._h(a.device.index)
    gh = np.ascontiguousarray(g.cpu().numpy()).view(np.float32).reshape(-1)
    h.call("qs_apply_2q", E._ptr(a), 9, gh.ctypes.data_as(C.POINTER(C.c_float)), 7, 2)
    h.call("qs_apply_2q_dev", E._ptr(b), 9, C.c_void_p(g.data_ptr()), 7, 2)
    assert np.array_equal(_bits(a), _bits(b))


def test_mcgate_device_equals_host_and_x_is_exact():
    u = bk.random_unitary().contiguous()
    a, b = _state(8, 3), _state(8, 3)
    bk.apply_mcgate(a, u, [1, 6], 3)
    bk.apply_mcgate(b, u.cpu(), [1, 6], 3)
    assert np.array_equal(_bits(a), _bits(b))
    x = bk.pauli_x_gate()
    before = a.cpu().numpy()
    bk.apply_mcgate(a, x, [2], 5)
    after = a.cpu().numpy()
    idx = np.arange(256)
    sel = (idx >> 2) & 1 == 1
    expect = before.copy()
    expect[sel] = before[idx[sel] ^ (1 << 5)]
    assert np.array_equal(after, expect)


def test_host_pointer_rejected():
    a = _state(4, 4)
    host = np.eye(2, dtype=np.complex64)
    with pytest.raises(_lib.QsimError, match="device memory"):
        E._h(a.device.index).call("qs_apply_1q_dev", E._ptr(a), 4, C.c_void_p(host.ctypes.data), 0)
