"""Torch-tensor kernel API, call-compatible with the reference's
bwk/python/blackwell_kernels/cuquantum.py (same names, argument meaning,
in-place mutation and return values), backed by libqsim.so.

Differences, by design:
* gate matrices may live on either device; they are read on the host and
  passed to the kernel by value (the reference reads a device tensor);
* ``sample`` draws FP64 uniforms and searches an FP64 CDF (the reference's
  FP32 CDF loses resolution beyond ~2^24 amplitudes, sample_sm120.cu:109-123);
* reductions accumulate in FP64 in a fixed order (no float atomics);
* 64-bit indexing: states up to 2^34 amplitudes.
"""
from __future__ import annotations

import cmath
import ctypes as C
import math

import numpy as np
import torch

from qsim_b200 import _lib
from qsim_b200 import engine as E
from qsim_b200.engine import _h, _ptr, check_state

_C64 = torch.complex64


def _fast_args(state, gate, shape):
    """(extension, handle, n, state pointer, gate pointer) for a direct call
    into libqsim when state and gate are contiguous complex64 CUDA tensors on
    one device and the gate has `shape`; None otherwise (the general path then
    checks the arguments and reports what is wrong)."""
    F = _lib.fast()
    if F is None or type(state) is not torch.Tensor or type(gate) is not torch.Tensor:
        return None
    if not state.is_cuda or state.dtype != _C64 or gate.dtype != _C64 or gate.shape != shape:
        return None
    dev = state.get_device()
    if gate.get_device() != dev or not state.is_contiguous() or not gate.is_contiguous():
        return None
    N = state.numel()
    if N < 2 or N & (N - 1):
        return None
    return F, E._hptr(dev), N.bit_length() - 1, state.data_ptr(), gate.data_ptr()


def _gate_host(gate, shape) -> np.ndarray:
    if isinstance(gate, torch.Tensor):
        g = gate.detach().to("cpu", torch.complex64).contiguous().numpy()
    else:
        g = np.asarray(gate, dtype=np.complex64)
    if g.shape != shape:
        raise RuntimeError(f"gate must be {'x'.join(map(str, shape))}")
    return np.ascontiguousarray(g.view(np.float32).reshape(-1))


def _gate_dev(gate, shape, state: torch.Tensor):
    """A gate that is already a complex64 CUDA tensor of the right shape on
    the state's device, made contiguous (a device copy if needed), else None.
    The caller passes its data_ptr() while holding the tensor, so the memory
    stays allocated until the gate kernel is queued; after that torch reuses
    it only for work queued later on the stream.  The kernel reads the gate
    itself: no host copy, no stream synchronisation."""
    if (isinstance(gate, torch.Tensor) and gate.is_cuda and gate.dtype == torch.complex64
            and tuple(gate.shape) == shape and gate.device == state.device):
        return gate if gate.is_contiguous() else gate.contiguous()
    return None


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _ints(x) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        x = x.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(x, dtype=np.int64).reshape(-1).astype(np.int32))


# ------------------------------------------------------------------- gates
def apply_gate(state: torch.Tensor, gate: torch.Tensor, target_qubit: int) -> torch.Tensor:
    """Single-qubit gate in place (cuquantum.py:40-51)."""
    a = _fast_args(state, gate, (2, 2))
    if a is not None:
        a[0].apply_1q_dev(a[1], a[3], a[2], a[4], int(target_qubit))
        return state
    n = check_state(state)
    gd = _gate_dev(gate, (2, 2), state)
    if gd is not None:
        _h(state.get_device()).call("qs_apply_1q_dev", state.data_ptr(), n, gd.data_ptr(), int(target_qubit))
        return state
    g = _gate_host(gate, (2, 2))
    _h(state.device.index).call("qs_apply_1q", _ptr(state), n, _fp(g), int(target_qubit))
    return state


def apply_gate_2q(state: torch.Tensor, gate: torch.Tensor, qubit0: int, qubit1: int) -> torch.Tensor:
    """Two-qubit gate in place (cuquantum.py:54-66).  As in the reference
    (apply_gate2q_sm120.cu:244-247) bit 0 of the 4x4 index is min(q0, q1)."""
    if qubit0 == qubit1:
        raise RuntimeError("qubit0 and qubit1 must differ")
    lo, hi = min(qubit0, qubit1), max(qubit0, qubit1)
    a = _fast_args(state, gate, (4, 4))
    if a is not None:
        a[0].apply_2q_dev(a[1], a[3], a[2], a[4], int(lo), int(hi))
        return state
    n = check_state(state)
    gd = _gate_dev(gate, (4, 4), state)
    if gd is not None:
        _h(state.get_device()).call("qs_apply_2q_dev", state.data_ptr(), n, gd.data_ptr(), int(lo), int(hi))
        return state
    g = _gate_host(gate, (4, 4))
    _h(state.device.index).call("qs_apply_2q", _ptr(state), n, _fp(g), int(lo), int(hi))
    return state


def apply_gates_fused(state: torch.Tensor, gates: torch.Tensor, targets: torch.Tensor) -> torch.Tensor:
    """K 1Q gates in one fused program (cuquantum.py:69-80)."""
    F = _lib.fast()
    if (F is not None and type(state) is torch.Tensor and type(gates) is torch.Tensor
            and type(targets) is torch.Tensor and state.is_cuda and state.dtype == _C64
            and gates.dtype == _C64 and targets.dtype == torch.int32 and gates.dim() == 3
            and targets.dim() == 1 and state.is_contiguous() and gates.is_contiguous()
            and targets.is_contiguous()):
        # the common case in the fewest tensor queries: contiguous complex64
        # gates and int32 targets already on the state's device
        dev = state.get_device()
        N = state.numel()
        K = targets.shape[0]
        tp = targets.data_ptr()
        if (gates.get_device() == dev and targets.get_device() == dev and gates.shape[0] == K
                and gates.shape[1] == 2 and gates.shape[2] == 2 and N >= 2 and not (N & (N - 1))
                and not (tp & 7)):
            F.apply_gates_fused_dev(E._hptr(dev), state.data_ptr(), N.bit_length() - 1, gates.data_ptr(), tp, K)
            return state
    n = check_state(state)
    if (isinstance(gates, torch.Tensor) and isinstance(targets, torch.Tensor) and gates.is_cuda
            and gates.device == state.device and targets.device == state.device):
        # device tensors: the kernel reads matrices and targets itself (no host
        # copy, no stream synchronisation); one launch per 12 gates
        g = gates.detach()
        if g.dtype != _C64:
            g = g.to(_C64)
        if g.ndim != 3 or tuple(g.shape[1:]) != (2, 2):
            raise RuntimeError("gates must be [N, 2, 2]")
        t = targets.detach().reshape(-1)
        if t.numel() != g.shape[0]:
            raise RuntimeError("targets must have N entries")
        if t.dtype != torch.int32:
            t = t.to(torch.int32)
        g = g.contiguous()
        t = t.contiguous()
        if t.data_ptr() & 7:
            t = t.clone()
        dev = state.get_device()
        F = _lib.fast()
        if F is not None:
            F.apply_gates_fused_dev(E._hptr(dev), state.data_ptr(), n, g.data_ptr(), t.data_ptr(), int(t.numel()))
        else:
            _h(dev).call("qs_apply_gates_fused_dev", state.data_ptr(), n, g.data_ptr(), t.data_ptr(), int(t.numel()))
        return state
    if isinstance(gates, torch.Tensor):
        g = gates.detach().to("cpu", torch.complex64).contiguous().numpy()
    else:
        g = np.asarray(gates, dtype=np.complex64)
    if g.ndim != 3 or g.shape[1:] != (2, 2):
        raise RuntimeError("gates must be [N, 2, 2]")
    t = _ints(targets)
    if t.size != g.shape[0]:
        raise RuntimeError("targets must have N entries")
    gf = np.ascontiguousarray(g.view(np.float32).reshape(-1))
    _h(state.device.index).call("qs_apply_gates_fused", _ptr(state), n, _fp(gf), _ip(t), int(t.size))
    return state


def apply_gates_reg_tiled(state: torch.Tensor, gates: torch.Tensor, targets: torch.Tensor) -> torch.Tensor:
    """Low-qubit fused 1Q gates (cuquantum.py:83-98); any targets are accepted
    here, since the tile-pass engine is not limited to qubits 0-4."""
    return apply_gates_fused(state, gates, targets)


def apply_diagonal(state: torch.Tensor, diag: torch.Tensor, target_qubit: int) -> torch.Tensor:
    a = _fast_args(state, diag, (2,))
    if a is not None:
        a[0].apply_diag1_dev(a[1], a[3], a[2], a[4], int(target_qubit))
        return state
    n = check_state(state)
    dd = _gate_dev(diag, (2,), state)
    if dd is not None:
        _h(state.get_device()).call("qs_apply_diag1_dev", state.data_ptr(), n, dd.data_ptr(), int(target_qubit))
        return state
    d = _gate_host(diag, (2,))
    _h(state.device.index).call("qs_apply_diag1", _ptr(state), n, _fp(d), int(target_qubit))
    return state


def apply_diagonal_phase(state: torch.Tensor, phase: complex, target_qubit: int) -> torch.Tensor:
    """Multiply the bit=1 amplitudes of target_qubit by phase (half traffic)."""
    phase = complex(phase)
    F = _lib.fast()
    if F is not None and type(state) is torch.Tensor and state.is_cuda and state.dtype == _C64 \
            and state.is_contiguous():
        N = state.numel()
        if N >= 2 and not N & (N - 1):
            F.apply_phase(E._hptr(state.get_device()), state.data_ptr(), N.bit_length() - 1, phase.real, phase.imag,
                          int(target_qubit))
            return state
    n = check_state(state)
    _h(state.device.index).call("qs_apply_phase", _ptr(state), n, C.c_float(phase.real), C.c_float(phase.imag),
                                int(target_qubit))
    return state


def apply_diagonal_2q(state: torch.Tensor, diag: torch.Tensor, qubit0: int, qubit1: int) -> torch.Tensor:
    a = _fast_args(state, diag, (4,))
    if a is not None:
        a[0].apply_diag2_dev(a[1], a[3], a[2], a[4], int(qubit0), int(qubit1))
        return state
    n = check_state(state)
    dd = _gate_dev(diag, (4,), state)
    if dd is not None:
        _h(state.get_device()).call("qs_apply_diag2_dev", state.data_ptr(), n, dd.data_ptr(), int(qubit0), int(qubit1))
        return state
    d = _gate_host(diag, (4,))
    _h(state.device.index).call("qs_apply_diag2", _ptr(state), n, _fp(d), int(qubit0), int(qubit1))
    return state


def state_init(n_qubits: int) -> torch.Tensor:
    return E.state_init(n_qubits, "cuda")


def _is_x(g: np.ndarray) -> bool:
    return np.array_equal(g.view(np.complex64).reshape(2, 2), np.array([[0, 1], [1, 0]], dtype=np.complex64))


def _is_swap(g: np.ndarray) -> bool:
    return np.array_equal(g.view(np.complex64).reshape(4, 4), np.eye(4, dtype=np.complex64)[[0, 2, 1, 3]])


def apply_mcgate(state: torch.Tensor, gate: torch.Tensor, controls, target_qubit: int) -> torch.Tensor:
    """Multi-controlled 2x2 (cuquantum.py:297-317); an exact X moves values."""
    a = _fast_args(state, gate, (2, 2))
    if a is not None and isinstance(controls, (list, tuple)):
        a[0].apply_mc1q_dev(a[1], a[3], a[2], a[4], controls, int(target_qubit))
        return state
    n = check_state(state)
    c = _ints(controls)
    if c.size > 7:
        raise RuntimeError("controls must have 0-7 elements")
    h = _h(state.device.index)
    gd = _gate_dev(gate, (2, 2), state)
    if gd is not None:
        # the matrix stays on the device; an X there is still exact (the
        # compensated 2x2 product of 0s and 1s rounds nothing)
        h.call("qs_apply_mc1q_dev", state.data_ptr(), n, gd.data_ptr(), _ip(c), int(c.size), int(target_qubit))
        return state
    g = _gate_host(gate, (2, 2))
    if _is_x(g):
        h.call("qs_apply_mcx", _ptr(state), n, _ip(c), int(c.size), int(target_qubit))
    else:
        h.call("qs_apply_mc1q", _ptr(state), n, _fp(g), _ip(c), int(c.size), int(target_qubit))
    return state


def apply_mc2qgate(state: torch.Tensor, gate: torch.Tensor, controls, target0: int, target1: int) -> torch.Tensor:
    """Multi-controlled 4x4 (cuquantum.py:320-337); bit 0 = min(target0, target1)."""
    a = _fast_args(state, gate, (4, 4))
    if a is not None and isinstance(controls, (list, tuple)):
        a[0].apply_mc2q_dev(a[1], a[3], a[2], a[4], controls, int(target0), int(target1))
        return state
    n = check_state(state)
    c = _ints(controls)
    if c.size > 7:
        raise RuntimeError("controls must have 0-7 elements")
    h = _h(state.device.index)
    gd = _gate_dev(gate, (4, 4), state)
    if gd is not None:
        # read on the device (a SWAP there is still exact: 0/1 products)
        h.call("qs_apply_mc2q_dev", state.data_ptr(), n, gd.data_ptr(), _ip(c), int(c.size), int(target0),
               int(target1))
        return state
    g = _gate_host(gate, (4, 4))
    if _is_swap(g):
        h.call("qs_apply_mcswap", _ptr(state), n, _ip(c), int(c.size), int(target0), int(target1))
    else:
        h.call("qs_apply_mc2q", _ptr(state), n, _fp(g), _ip(c), int(c.size), int(target0), int(target1))
    return state


# ------------------------------------------------------------ reductions
def measure_qubit(state: torch.Tensor, target_qubit: int, random_val: float) -> int:
    return E.measure(state, target_qubit, random_val)


def measure_probs(state: torch.Tensor) -> torch.Tensor:
    return E.probs(state)


def sample(state: torch.Tensor, n_shots: int) -> torch.Tensor:
    """n_shots basis indices drawn from |state|^2 (cuquantum.py:283-294)."""
    return E.sample(state, n_shots)


def expectation_z(state: torch.Tensor, z_mask: int) -> float:
    n = check_state(state)
    out = C.c_double()
    _h(state.device.index).call("qs_expect_z", _ptr(state), n, C.c_uint64(int(z_mask)), C.byref(out))
    return float(out.value)


def expectation_pauli(state: torch.Tensor, z_mask: int, xy_qubit: int, op: int) -> float:
    """<Z-string x (X or Y on xy_qubit)> (cuquantum.py:472-487); op 0 = Z only,
    1 = X, 2 = Y.  (libqsim also evaluates arbitrary multi-X/Y strings.)"""
    if op not in (0, 1, 2):
        raise RuntimeError("op must be 0=I/Z, 1=X, 2=Y")
    if op == 0:
        return expectation_z(state, z_mask)
    from qsim_b200.paulis import PauliSum
    x = 1 << int(xy_qubit)
    z = int(z_mask) | (x if op == 2 else 0)
    n = check_state(state)
    return E.expect_pauli_sum(state, PauliSum([x], [z], [1.0], n))


def renormalize(state: torch.Tensor) -> torch.Tensor:
    return E.renormalize(state)


# ----------------------------------------------------------------- batch
def apply_gate_batched(states: torch.Tensor, gate: torch.Tensor, target_qubit: int) -> torch.Tensor:
    if states.dim() != 2 or not states.is_cuda or states.dtype != torch.complex64 or not states.is_contiguous():
        raise RuntimeError("states must be a contiguous complex64 CUDA tensor [N, 2^n]")
    N, m = states.shape
    n = m.bit_length() - 1
    g = _gate_host(gate, (2, 2))
    _h(states.device.index).call("qs_apply_1q_batched", _ptr(states), int(N), n, _fp(g), int(target_qubit))
    return states


def apply_gates_batched_fused(states: torch.Tensor, gates: torch.Tensor, targets: torch.Tensor) -> torch.Tensor:
    if states.dim() != 2 or not states.is_cuda or states.dtype != torch.complex64 or not states.is_contiguous():
        raise RuntimeError("states must be a contiguous complex64 CUDA tensor [N, 2^n]")
    N, m = states.shape
    n = m.bit_length() - 1
    g = gates.detach().to("cpu", torch.complex64).contiguous().numpy() if isinstance(gates, torch.Tensor) \
        else np.asarray(gates, dtype=np.complex64)
    t = _ints(targets)
    gf = np.ascontiguousarray(g.view(np.float32).reshape(-1))
    _h(states.device.index).call("qs_apply_gates_batched_fused", _ptr(states), int(N), n, _fp(gf), _ip(t),
                                 int(t.size))
    return states


def state_init_batched(n_states: int, n_qubits: int) -> torch.Tensor:
    s = torch.empty(int(n_states), 1 << int(n_qubits), dtype=torch.complex64, device="cuda")
    _h(s.device.index).call("qs_state_init_batched", _ptr(s), int(n_states), int(n_qubits))
    return s


class CircuitGraph:
    """CUDA-graph capture of a list of 1Q gates (cuquantum.py:101-130).  libqsim
    launches on torch's current stream, so the capture records them."""

    def __init__(self, state: torch.Tensor, gates: torch.Tensor, targets):
        if isinstance(targets, torch.Tensor):
            targets = targets.tolist()
        self._gates = [_gate_host(gates[i], (2, 2)) for i in range(len(targets))]
        self._targets = [int(t) for t in targets]
        for g, t in zip(gates, targets):
            apply_gate(state, g, int(t))
        torch.cuda.synchronize()
        self._graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self._graph):
            for g, t in zip(gates, targets):
                apply_gate(state, g, int(t))
        self._state = state

    def replay(self):
        self._graph.replay()


# ----------------------------------------------------------- Chebyshev
def spmv_csr(row_ptr, col_idx, values, x, y, alpha_re=1.0, alpha_im=0.0, beta_re=0.0, beta_im=0.0):
    """y = alpha*A*x + beta*y (cuquantum.py:518-531)."""
    for t, name in ((row_ptr, "row_ptr"), (col_idx, "col_idx"), (values, "values"), (x, "x"), (y, "y")):
        if not t.is_cuda:
            raise RuntimeError(f"{name} must be a CUDA tensor")
    if row_ptr.dtype != torch.int32 or col_idx.dtype != torch.int32:
        raise RuntimeError("row_ptr/col_idx must be int32")
    if values.dtype != torch.complex64 or x.dtype != torch.complex64 or y.dtype != torch.complex64:
        raise RuntimeError("values, x and y must be complex64")
    _h(x.device.index).call("qs_spmv_csr", _ptr(row_ptr), _ptr(col_idx), _ptr(values), int(row_ptr.numel() - 1),
                            _ptr(x), _ptr(y), float(alpha_re), float(alpha_im), float(beta_re), float(beta_im))


def chebyshev_step(spmv_result, t_prev, t_next):
    _h(t_next.device.index).call("qs_cheb_step", _ptr(spmv_result), _ptr(t_prev), _ptr(t_next),
                                 int(spmv_result.numel()))


def chebyshev_accum(accum, t_k, c_re, c_im):
    _h(accum.device.index).call("qs_cheb_accum", _ptr(accum), _ptr(t_k), float(c_re), float(c_im),
                                int(accum.numel()))


def chebyshev_step_accum(spmv_result, t_prev, t_next, accum, c_re, c_im):
    _h(accum.device.index).call("qs_cheb_step_accum", _ptr(spmv_result), _ptr(t_prev), _ptr(t_next), _ptr(accum),
                                float(c_re), float(c_im), int(accum.numel()))


# ------------------------------------------------------ gate constructors
def hadamard_gate(device="cuda"):
    return torch.tensor([[1, 1], [1, -1]], dtype=torch.complex64, device=device) / (2 ** 0.5)


def pauli_x_gate(device="cuda"):
    return torch.tensor([[0, 1], [1, 0]], dtype=torch.complex64, device=device)


def cnot_gate(device="cuda"):
    """|00>->|00>, |01>->|01>, |10>->|11>, |11>->|10> (control in index bit 1)."""
    return torch.tensor([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=torch.complex64,
                        device=device)


def cz_gate(device="cuda"):
    return torch.tensor([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, -1]], dtype=torch.complex64,
                        device=device)


def swap_gate(device="cuda"):
    return torch.tensor([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=torch.complex64,
                        device=device)


def cswap_gate(device="cuda"):
    return swap_gate(device)


def _haar(dim, device):
    z = torch.randn(dim, dim, dtype=torch.complex64)
    q, r = torch.linalg.qr(z)
    d = torch.diagonal(r)
    return (q * (d / d.abs()).unsqueeze(0)).contiguous().to(device)


def random_unitary(device="cuda"):
    return _haar(2, device)


def random_unitary_4x4(device="cuda"):
    return _haar(4, device)


def rz_gate_diag(theta, device="cuda"):
    return torch.tensor([cmath.exp(-1j * theta / 2), cmath.exp(1j * theta / 2)], dtype=torch.complex64,
                        device=device)


def phase_gate_diag(theta, device="cuda"):
    return torch.tensor([1.0, cmath.exp(1j * theta)], dtype=torch.complex64, device=device)


def t_gate_diag(device="cuda"):
    return torch.tensor([1.0, cmath.exp(1j * math.pi / 4)], dtype=torch.complex64, device=device)


def s_gate_diag(device="cuda"):
    return torch.tensor([1.0, 1j], dtype=torch.complex64, device=device)


def z_gate_diag(device="cuda"):
    return torch.tensor([1.0, -1.0], dtype=torch.complex64, device=device)


def cz_gate_diag(device="cuda"):
    return torch.tensor([1.0, 1.0, 1.0, -1.0], dtype=torch.complex64, device=device)


# ------------------------------------------------------------------ noise
# cuquantum.py:352-411 / noise_sm120.cu:238-373: one channel on one state,
# random_val drawn with torch.rand when not given, branch code returned.
def _noise(entry: str, state: torch.Tensor, target_qubit: int, prob: float, random_val) -> int:
    n = check_state(state)
    if random_val is None:
        random_val = torch.rand(1).item()
    out = C.c_int32(0)
    _h(state.device.index).call(entry, _ptr(state), n, int(target_qubit), float(prob), float(random_val),
                                C.byref(out))
    return int(out.value)


def apply_depolarizing(state: torch.Tensor, target_qubit: int, p: float, random_val: float = None) -> int:
    """Identity w.p. 1-p, else Pauli X / Y / Z w.p. p/3 each; returns 0..3."""
    return _noise("qs_apply_depolarizing", state, target_qubit, p, random_val)


def apply_amplitude_damping(state: torch.Tensor, target_qubit: int, gamma: float, random_val: float = None) -> int:
    """T1 decay: returns 1 when the decay branch E1 was taken, else 0.  The
    jump branch is E1 = [[0, sqrt(gamma)], [0, 0]] exactly (the reference's
    kernel keeps the |0> amplitudes there, noise_sm120.cu:200-204)."""
    return _noise("qs_apply_amplitude_damping", state, target_qubit, gamma, random_val)


def apply_dephasing(state: torch.Tensor, target_qubit: int, lam: float, random_val: float = None) -> int:
    """T2 dephasing: returns 1 when the error branch E1 was taken, else 0."""
    return _noise("qs_apply_dephasing", state, target_qubit, lam, random_val)
