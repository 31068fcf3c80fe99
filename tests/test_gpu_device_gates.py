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


def test_diag2_and_mc2q_device_equal_host_and_swap_is_exact():
    rng = np.random.default_rng(5)
    d = torch.from_numpy(np.exp(1j * rng.uniform(0, 6.28, 4)).astype(np.complex64)).cuda()
    a, b = _state(9, 6), _state(9, 6)
    bk.apply_diagonal_2q(a, d, 7, 2)
    bk.apply_diagonal_2q(b, d.cpu(), 7, 2)
    assert np.array_equal(_bits(a), _bits(b))
    u = bk.random_unitary_4x4().contiguous()
    bk.apply_mc2qgate(a, u, [1, 4], 6, 0)
    bk.apply_mc2qgate(b, u.cpu(), [1, 4], 6, 0)
    assert np.array_equal(_bits(a), _bits(b))
    sw = torch.eye(4, dtype=torch.complex64, device="cuda")[[0, 2, 1, 3]].contiguous()
    before = a.cpu().numpy()
    bk.apply_mc2qgate(a, sw, [8], 3, 5)              # controlled SWAP on the device: values move exactly
    after = a.cpu().numpy()
    idx = np.arange(512)
    swap = ((idx >> 8) & 1 == 1) & (((idx >> 3) & 1) != ((idx >> 5) & 1))
    expect = before.copy()
    expect[swap] = before[idx[swap] ^ ((1 << 3) | (1 << 5))]
    assert np.array_equal(after, expect)


def test_host_pointer_rejected():
    a = _state(4, 4)
    host = np.eye(2, dtype=np.complex64)
    with pytest.raises(_lib.QsimError, match="device memory"):
        E._h(a.device.index).call("qs_apply_1q_dev", E._ptr(a), 4, C.c_void_p(host.ctypes.data), 0)


def _fused_ref(psi, gates, targets):
    """FP64: the 1Q gates applied one after another."""
    import sv_oracle as O
    from qsim_b200.circuit import Circuit, lower
    n = int(psi.size).bit_length() - 1
    qc = Circuit(n)
    for g, t in zip(gates, targets):
        qc.unitary(np.asarray(g, dtype=np.complex128), [int(t)])
    return O.simulate(n, lower(qc), psi.astype(np.complex128))


def test_fused_gates_device_and_host_inputs_and_repeats():
    """apply_gates_fused with CUDA gate/target tensors (one device launch)
    and with host arrays (the planner's fused plan, cached) agree with the
    FP64 oracle; calling the host form again with the same gates reuses the
    plan (the result equals fresh applications), and new gate values on the
    same targets are not served a stale plan."""
    n = 12
    gates = torch.stack([bk.random_unitary() for _ in range(10)]).contiguous()
    targets = torch.arange(10, dtype=torch.int32, device="cuda")
    a, b = _state(n, 5), _state(n, 5)
    psi0 = a.cpu().numpy()
    bk.apply_gates_fused(b, gates, targets)
    bk.apply_gates_fused(a, gates.cpu(), targets.cpu().tolist())
    assert np.abs(a.cpu().numpy() - b.cpu().numpy()).max() < 1e-5
    g_h = gates.cpu().numpy()
    ref = _fused_ref(psi0, g_h, range(10))
    assert np.abs(a.cpu().numpy() - ref).max() < 1e-5
    for _ in range(3):                                  # cache hits
        bk.apply_gates_fused(a, gates.cpu(), targets.cpu().tolist())
    ref2 = ref
    for _ in range(3):
        ref2 = _fused_ref(ref2.astype(np.complex64), g_h, range(10))
    assert np.abs(a.cpu().numpy() - ref2).max() < 1e-4
    gates2 = torch.stack([bk.random_unitary() for _ in range(10)]).contiguous()
    c = _state(n, 5)
    bk.apply_gates_fused(c, gates2.cpu(), targets.cpu().tolist())
    ref3 = _fused_ref(psi0, gates2.cpu().numpy(), range(10))
    assert np.abs(c.cpu().numpy() - ref3).max() < 1e-5
    # another stream: built afresh there, same bits
    d = _state(n, 5)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        bk.apply_gates_fused(d, gates2.cpu(), targets.cpu().tolist())
    s.synchronize()
    assert np.array_equal(_bits(c), _bits(d))


@pytest.mark.parametrize("n,k", [(1, 3), (5, 12), (12, 1), (13, 13), (16, 30), (20, 10)])
def test_fused_device_equals_single_gate_calls(n, k):
    """The device-tensor form of apply_gates_fused (qs_apply_gates_fused_dev:
    tiles holding the targets, gates applied in order in shared memory, one
    launch per 12 gates) agrees with one apply_gate call per gate (FMA chains
    against compensated products: ~1e-7 relative per gate) and with the FP64
    oracle, repeated targets and more gates than a launch takes included."""
    rng = np.random.default_rng(100 + n + k)
    tg = rng.integers(0, n, size=k)
    if k > 2:
        tg[1] = tg[0]                                      # a repeated target
    gates = torch.stack([bk.random_unitary() for _ in range(k)]).contiguous()
    targets = torch.from_numpy(tg.astype(np.int64)).cuda()  # int64 is converted on the device
    a, b = _state(n, 7), _state(n, 7)
    psi0 = a.cpu().numpy()
    bk.apply_gates_fused(a, gates, targets)
    for j in range(k):
        bk.apply_gate(b, gates[j], int(tg[j]))
    scale = np.abs(b.cpu().numpy()).max()
    assert np.abs(a.cpu().numpy() - b.cpu().numpy()).max() <= 1e-6 * k * scale
    ref = _fused_ref(psi0, gates.cpu().numpy(), tg)
    assert np.abs(a.cpu().numpy() - ref).max() < 1e-5 * max(1, k) ** 0.5
    code = C.c_int(-1)
    E._h(a.device.index).call("qs_device_status", C.byref(code))
    assert code.value == 0


def test_fused_device_target_out_of_range_sets_status():
    """A target outside the state, found on the device: the launch leaves the
    state as it was and reports bit 16 through qs_device_status."""
    n = 10
    gates = torch.stack([bk.random_unitary() for _ in range(3)]).contiguous()
    for bad in (n, -1):
        a = _state(n, 8)
        before = _bits(a).copy()
        targets = torch.tensor([0, bad, 2], dtype=torch.int32, device="cuda")
        bk.apply_gates_fused(a, gates, targets)
        code = C.c_int(-1)
        E._h(a.device.index).call("qs_device_status", C.byref(code))
        assert code.value == 16
        assert np.array_equal(_bits(a), before)
    E._h(a.device.index).call("qs_device_status", C.byref(code))
    assert code.value == 0


def test_run_circuit_cache_many_circuits():
    """More distinct circuits than the handle keeps: every call still runs
    its own circuit (evictions free programs without disturbing later runs)."""
    import sv_oracle as O
    from qsim_b200 import workloads as W
    h = E._h(0)
    n = 10
    outs = []
    for rep in range(2):
        # the second sweep, in reverse, hits the 16 kept plans, then evicts
        for seed in (range(20) if rep == 0 else reversed(range(20))):
            ops = W.qv_ops(n, 4, seed=seed)
            st = torch.zeros(1 << n, dtype=torch.complex64, device="cuda")
            st[0] = 1
            h.call("qs_run_circuit", E._ptr(st), n, ops.ctypes.data_as(C.POINTER(_lib.QsOp)), len(ops))
            outs.append((seed, st))
    torch.cuda.synchronize()
    first = {}
    for seed, st in outs:
        ref = O.simulate(n, W.qv_ops(n, 4, seed=seed))
        assert abs(1 - O.fidelity(st.cpu().numpy(), ref)) <= 1e-6
        if seed in first:
            assert np.array_equal(_bits(st), _bits(first[seed]))
        first[seed] = st
