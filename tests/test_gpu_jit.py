"""Specialised tile passes (NVRTC) against the generic pass kernel and the
FP64 oracle: the specialised kernels must return the interpreter's
amplitudes bit for bit, for every device-op kind, tile width and
register-block width, from a given state and from |0..0>."""
import time

import numpy as np
import pytest
import torch

import sv_oracle as O
from qsim_b200 import engine as E
from qsim_b200 import workloads as W
from test_oracle_golden import _random_ops

pytestmark = pytest.mark.gpu


def _run(n, ops, mode, psi0=None, tile_bits=0, block_bits=0):
    h = E._h()
    h.call("qs_set_tile_bits", tile_bits)
    h.call("qs_set_block_bits", block_bits)
    h.call("qs_set_tensor_cores", 0)   # every pass on the kernels under comparison
    E.set_jit(mode)
    try:
        plan = E.Plan(n, ops)
        s = E.empty_state(n)
        if psi0 is None:
            plan.execute_from_zero(s)
        else:
            s.copy_(torch.from_numpy(psi0))
            plan.execute(s)
        torch.cuda.synchronize()
        return s.cpu().numpy(), plan.refresh_info()
    finally:
        E.set_jit(1)
        h.call("qs_set_tile_bits", 0)
        h.call("qs_set_block_bits", 0)
        h.call("qs_set_tensor_cores", 1)


def _same_bits(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("kak", ["0", "1"])
@pytest.mark.parametrize("n,tile_bits,block_bits", [(6, 10, 5), (13, 10, 4), (15, 12, 3), (17, 13, 5),
                                                    (18, 14, 5), (17, 10, 2)])
def test_random_all_kinds_bit_identical(n, tile_bits, block_bits, kak, monkeypatch):
    # the same plan (Cartan split of dense 2Q gates forced on or off) on both kernels
    monkeypatch.setenv("QSIM_KAK", kak)
    rng = np.random.default_rng(5000 + n)
    ops = _random_ops(n, 100, rng)
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi0 = (psi0 / np.linalg.norm(psi0)).astype(np.complex64)
    ref, info0 = _run(n, ops, 0, psi0, tile_bits, block_bits)
    got, info2 = _run(n, ops, 2, psi0, tile_bits, block_bits)
    assert info0["n_jit_passes"] == 0
    assert info2["n_jit_passes"] == info2["n_passes"] >= 1
    assert _same_bits(ref, got)
    exact = O.simulate(n, ops, psi0.astype(np.complex128))
    assert abs(1 - O.fidelity(got, exact)) <= 1e-6


@pytest.mark.parametrize("tile_bits,block_bits", [(10, 5), (13, 4), (13, 5)])
def test_layers_from_zero_bit_identical(tile_bits, block_bits):
    ops = W.layers_ops(20, 8, seed=3)
    ref, _ = _run(20, ops, 0, None, tile_bits, block_bits)
    got, info = _run(20, ops, 2, None, tile_bits, block_bits)
    assert info["n_jit_passes"] == info["n_passes"] > 1
    assert _same_bits(ref, got)
    assert abs(1 - O.fidelity(got, O.simulate(20, ops))) <= 1e-6


@pytest.mark.parametrize("kak", ["0", "1"])
def test_qv_bit_identical(kak, monkeypatch):
    monkeypatch.setenv("QSIM_KAK", kak)
    ops = W.qv_ops(14, 14, 7)
    ref, _ = _run(14, ops, 0, None, 0, 5)    # same register-block width on both kernels
    got, info = _run(14, ops, 2, None, 0, 5)
    assert info["n_jit_passes"] == info["n_passes"]
    assert _same_bits(ref, got)
    assert abs(1 - O.fidelity(got, O.simulate(14, ops))) <= 1e-6


def test_tiered_mode_switches_over_and_matches():
    """Mode 1: plans below the qubit threshold stay on the generic kernel;
    above it the first execution starts a background compile and later
    executions switch to the specialised passes; a new plan of the same
    circuit finds every pass in the kernel cache at its first execution."""
    ops1 = W.layers_ops(16, 3, seed=11)
    ops2 = W.layers_ops(16, 3, seed=12)
    ref2, _ = _run(16, ops2, 0)
    s = E.empty_state(16)
    E.set_jit(1, 17)
    try:
        plan = E.Plan(16, ops1)
        plan.execute_from_zero(s)
        torch.cuda.synchronize()
        assert plan.refresh_info()["n_jit_passes"] == 0
        E.set_jit(1, 16)
        plan2 = E.Plan(16, ops2)
        deadline = time.time() + 300
        while True:
            plan2.execute_from_zero(s)
            torch.cuda.synchronize()
            if plan2.refresh_info()["n_jit_passes"] == plan2.info["n_passes"]:
                break
            assert time.time() < deadline, "background specialisation did not finish"
            time.sleep(0.2)
        assert _same_bits(ref2, s.cpu().numpy())
        plan3 = E.Plan(16, ops2)
        s.zero_()
        plan3.execute_from_zero(s)
        torch.cuda.synchronize()
        assert plan3.refresh_info()["n_jit_passes"] == plan3.info["n_passes"]
        assert _same_bits(ref2, s.cpu().numpy())
    finally:
        E.set_jit(1, 24)


@pytest.mark.parametrize("tile_bits", [12, 13])
def test_pipelined_passes_24_qubits_bit_identical(tile_bits):
    """24 qubits of the layered generator: tiles whose high qubits form up
    to ten runs (box dimensions plus boxes walked one by one), from |0..0>
    and from a given state, on the pipelined kernels (TMA stage ring) and
    the generic interpreter."""
    ops = W.layers_ops(24, 8, seed=5)
    ref, _ = _run(24, ops, 0, None, tile_bits, 5)
    got, info = _run(24, ops, 2, None, tile_bits, 5)
    assert info["n_jit_passes"] == info["n_passes"] > 3
    assert _same_bits(ref, got)
    rng = np.random.default_rng(8)
    psi0 = (rng.standard_normal(1 << 24) + 1j * rng.standard_normal(1 << 24)).astype(np.complex64)
    psi0 /= np.float32(np.linalg.norm(psi0))
    ref, _ = _run(24, ops, 0, psi0, tile_bits, 5)
    got, _ = _run(24, ops, 2, psi0, tile_bits, 5)
    assert _same_bits(ref, got)


def test_pipelined_pass_bounded_wait_reports_status():
    """The pipelined pass's waits are bounded: with its first tile's copy
    withheld (the test hook), the consumer and producer waits run out after
    50 ms, the status word reports both, and the handle keeps working."""
    import ctypes as C
    n = 20
    ops = W.layers_ops(n, 4, seed=9)
    h = E._h()
    E.set_jit(2)
    try:
        plan = E.Plan(n, ops)
        s = E.empty_state(n)
        plan.execute_from_zero(s)
        torch.cuda.synchronize()
        assert plan.refresh_info()["n_jit_passes"] == plan.info["n_passes"]
        code = C.c_int(-1)
        h.call("qs_device_status", C.byref(code))
        assert code.value == 0
        h.call("qs_set_wait_test", 1)
        plan.execute(s)                # the first pass loads: its first tile never arrives
        torch.cuda.synchronize()
        h.call("qs_device_status", C.byref(code))
        assert code.value == 3, code.value
        h.call("qs_device_status", C.byref(code))
        assert code.value == 0         # read and cleared
        plan.execute_from_zero(s)      # the context is usable and the result right
        torch.cuda.synchronize()
        assert abs(1 - O.fidelity(s.cpu().numpy(), O.simulate(n, ops))) <= 1e-6
        h.call("qs_device_status", C.byref(code))
        assert code.value == 0
    finally:
        E.set_jit(1, 24)
