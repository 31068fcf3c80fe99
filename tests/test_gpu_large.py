"""Maximum sizes: a 33-qubit state (2^33 complex64 = 64 GiB; the reference's
int32 indexing stops at 2^31 amplitudes) through the fused plan path: GHZ
preparation, amplitudes and norm checked analytically."""
import math

import numpy as np
import pytest
import torch

from qsim_b200 import engine as E
from qsim_b200.circuit import Circuit, lower

pytestmark = pytest.mark.gpu


def test_ghz_33_qubits():
    n = 33
    free, _ = torch.cuda.mem_get_info()
    if free < (8 << n) + (4 << 30):
        pytest.skip("not enough free HBM for a 64 GiB state")
    qc = Circuit(n)
    qc.h(0)
    for q in range(1, n):
        qc.cx(q - 1, q)
    torch.cuda.empty_cache()
    s = E.empty_state(n)
    try:
        E.Plan(n, lower(qc)).execute_from_zero(s)
        torch.cuda.synchronize()
        r = 1.0 / math.sqrt(2.0)
        ends = torch.stack([s[0], s[-1]]).cpu().numpy()
        assert np.allclose(ends, [r, r], atol=1e-7)
        # everything else is exactly zero: the norm is carried by the two ends
        assert abs(E.norm2(s) - 1.0) < 1e-6
        mid = s[1: 1 << 20].abs().max().item()
        assert mid == 0.0
    finally:
        del s
        torch.cuda.empty_cache()


def test_layers_32_qubits_pipelined_equals_interpreter():
    """The 32-qubit layered generator (6 layers with a Toffoli) on the
    pipelined specialised passes (TMA stage ring, two compute groups,
    ~3.5k tiles per CTA) and on the generic interpreter: the two 32 GiB
    states are bit-identical, and the norm is 1 (FP64 reduction)."""
    from qsim_b200 import workloads as W
    n = 32
    free, _ = torch.cuda.mem_get_info()
    if free < 2 * (8 << n) + (4 << 30):
        pytest.skip("not enough free HBM for two 32 GiB states")
    ops = W.layers_ops(n, 6, seed=1, toffoli_every=3)
    torch.cuda.empty_cache()
    a = E.empty_state(n)
    b = E.empty_state(n)
    h = E._h()
    try:
        h.call("qs_set_tile_bits", 13)       # the same plan shape on both kernels
        h.call("qs_set_block_bits", 5)
        E.set_jit(2)
        pa = E.Plan(n, ops)
        pa.execute_from_zero(a)
        torch.cuda.synchronize()
        assert pa.refresh_info()["n_jit_passes"] == pa.info["n_passes"] > 3
        E.set_jit(0)
        pb = E.Plan(n, ops)
        pb.execute_from_zero(b)
        torch.cuda.synchronize()
        assert pb.refresh_info()["n_jit_passes"] == 0
        import ctypes as C
        code = C.c_int(-1)
        h.call("qs_device_status", C.byref(code))
        assert code.value == 0
        assert torch.equal(a.view(torch.int64), b.view(torch.int64))
        assert abs(E.norm2(a) - 1.0) < 1e-5
    finally:
        E.set_jit(1, 24)
        h.call("qs_set_tile_bits", 0)
        h.call("qs_set_block_bits", 0)
        del a, b
        torch.cuda.empty_cache()
