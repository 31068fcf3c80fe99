"""The tensor-core tile pass (qs_pass_tc.cu): dense-4x4-only passes with
5-qubit register blocks and 12/13-qubit tiles applied as 32x32 block
matrices with tcgen05.mma (TF32, three-product high/low split, FP32
accumulator in tensor memory).  Every circuit must meet |1-F| <= 1e-6 and
the max-amplitude bound against the FP64 oracle, agree with the CUDA-core
interpreter to ~1e-6 relative, and leave the device status word clear."""
import ctypes as C

import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200 import engine as E
from qsim_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _batch(widths, oo, ops, so, tc):
    h = E._h()
    h.call("qs_set_tensor_cores", int(tc))
    try:
        bp = E.BatchPlan(widths, oo, ops, so)
        st = bp.alloc_states()
        bp.execute(st)
        bp.execute(st.zero_())   # the second execution captures the graph; same result
        torch.cuda.synchronize()
        code = C.c_int(-1)
        h.call("qs_device_status", C.byref(code))
        assert code.value == 0
        return bp.info, st.cpu().numpy()
    finally:
        h.call("qs_set_tensor_cores", 1)


@pytest.mark.parametrize("lo,hi,n", [(12, 16, 24), (17, 20, 8)])
def test_qv_batch_on_tensor_cores_vs_oracle_and_cuda_cores(lo, hi, n):
    widths, oo, ops, so = W.qv_batch(n, lo, hi, seed=70 + lo)
    info_tc, tc = _batch(widths, oo, ops, so, 1)
    info_cc, cc = _batch(widths, oo, ops, so, 0)
    assert info_tc["n_tc_launches"] > 0 and info_cc["n_tc_launches"] == 0
    for c in range(len(widths)):
        w = int(widths[c])
        got = tc[so[c]: so[c] + (1 << w)]
        ref = O.simulate(w, ops[oo[c]: oo[c + 1]])
        scale = np.abs(ref).max()
        assert abs(1 - O.fidelity(got, ref)) <= 1e-6, (c, w)
        assert abs(np.vdot(got, got).real - 1.0) <= 1e-5, (c, w)   # no drift of the norm
        assert np.abs(got - ref).max() <= 2e-5 * scale, (c, w)
        other = cc[so[c]: so[c] + (1 << w)]
        assert np.abs(got - other).max() <= 2e-5 * scale, (c, w)


def test_tensor_core_pass_is_deterministic():
    """Two executions of the same batch plan give the same bits (the MMA
    order and the accumulator are fixed)."""
    widths, oo, ops, so = W.qv_batch(6, 13, 18, seed=5)
    _, a = _batch(widths, oo, ops, so, 1)
    _, b = _batch(widths, oo, ops, so, 1)
    assert np.array_equal(a, b)


def test_twelve_qubit_tiles_many_tiles_per_circuit():
    """The tensor-core pass with 12-qubit tiles on circuits of 13-17 qubits
    (2 to 32 tiles per pass, one 128-group slice per block), the shape the
    autotuner may record for a width: every circuit against FP64."""
    widths, oo, ops, so = W.qv_batch(10, 13, 17, seed=91)
    dev = torch.cuda.current_device()
    L = E._h().L
    saved = {}
    tb, bb = C.c_int(0), C.c_int(0)
    for w in range(1, 41):
        if L.qs_autotune_get(dev, w, C.byref(tb), C.byref(bb)) == 0:
            saved[w] = (tb.value, bb.value)
    E.autotune_set({w: (12, 5) for w in range(13, 18)})
    try:
        info, st = _batch(widths, oo, ops, so, 1)
    finally:
        E.autotune_clear(dev)        # the table as it was before the test
        E.autotune_set(saved, dev)
    assert info["n_tc_launches"] > 0
    for c in range(len(widths)):
        w = int(widths[c])
        got = st[so[c]: so[c] + (1 << w)]
        ref = O.simulate(w, ops[oo[c]: oo[c + 1]])
        assert abs(1 - O.fidelity(got, ref)) <= 1e-6, (c, w)
        assert np.abs(got - ref).max() <= 2e-5 * np.abs(ref).max(), (c, w)
