"""Torch-facing engine over the C ABI.

States are ``torch.complex64`` CUDA tensors; their data pointers go straight
to libqsim, which runs on torch's current CUDA stream.  torch is used only for
device memory, streams and RNG here; every kernel that touches a state is in
libqsim.so.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._lib import QsBatchInfo, QsOp, QsPlanInfo
from .circuit import OP_DTYPE


def _record_use(plan) -> None:
    """Remember the last launch that reads the plan's device program (an
    event on the current stream), so destroying the plan waits for exactly
    that work instead of the whole device."""
    ev = torch.cuda.Event()
    ev.record(torch.cuda.current_stream(plan.device))
    plan._uses = getattr(plan, "_uses", [])[-7:] + [ev]


def _wait_uses(plan) -> None:
    for ev in getattr(plan, "_uses", []):
        ev.synchronize()


try:  # torch's current stream as a raw pointer, without building a Stream object per call
    _raw_stream = torch._C._cuda_getCurrentRawStream
except AttributeError:  # pragma: no cover - older torch
    _raw_stream = None


def _h(device: int | None = None) -> _lib.Handle:
    dev = torch.cuda.current_device() if device is None else int(device)
    sp = _raw_stream(dev) if _raw_stream is not None else torch.cuda.current_stream(dev).cuda_stream
    return _lib.handle(dev, sp)


def _hptr(device: int) -> int:
    """Raw qs_handle_t of this thread's handle on `device`, bound to torch's
    current stream there (for the direct per-gate calls)."""
    sp = _raw_stream(device) if _raw_stream is not None else torch.cuda.current_stream(device).cuda_stream
    return _lib.handle(device, sp).h.value


def autotune_batch(widths, op_offsets, ops, device: int | None = None) -> dict:
    """Tunes tile and register-block widths per circuit width on the given
    circuits (one sample per width); returns {width: (tile_bits, block_bits)}."""
    dev = torch.cuda.current_device() if device is None else int(device)
    widths = np.ascontiguousarray(widths, dtype=np.int32)
    op_offsets = np.ascontiguousarray(op_offsets, dtype=np.int64)
    ops, p = _ops_ptr(ops)
    h = _h(dev)
    h.call("qs_autotune_batch", int(len(widths)), C.c_void_p(widths.ctypes.data),
           C.c_void_p(op_offsets.ctypes.data), p)
    out = {}
    tb, bb = C.c_int(0), C.c_int(0)
    for w in sorted(set(int(x) for x in widths)):
        if h.L.qs_autotune_get(dev, w, C.byref(tb), C.byref(bb)) == 0:
            out[w] = (tb.value, bb.value)
    return out


def autotune_set(table: dict, device: int | None = None) -> None:
    """Records {width: (tile_bits, block_bits)} entries as autotune_batch
    would (a table saved from an earlier run, or a fixed shape)."""
    dev = torch.cuda.current_device() if device is None else int(device)
    L = _lib.load()
    for w, (tb, bb) in table.items():
        _lib.check(L.qs_autotune_set(dev, int(w), int(tb), int(bb)))


def autotune_clear(device: int | None = None) -> None:
    _lib.load().qs_autotune_clear(-1 if device is None else int(device))


def set_jit(mode: int, min_qubits: int = 0, device: int | None = None) -> None:
    """Pass specialisation for plans executed by this thread's handle:
    0 = never, 1 = plans on >= min_qubits qubits, 2 = every plan."""
    _h(device).call("qs_set_jit", int(mode), int(min_qubits))


def _ptr(t: torch.Tensor) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _ops_ptr(ops: np.ndarray):
    if ops.dtype != OP_DTYPE or not ops.flags["C_CONTIGUOUS"]:
        ops = np.ascontiguousarray(ops, dtype=OP_DTYPE)
    return ops, ops.ctypes.data_as(C.POINTER(QsOp))


def check_state(state: torch.Tensor) -> int:
    if not isinstance(state, torch.Tensor) or not state.is_cuda:
        raise RuntimeError("state must be CUDA")
    if state.dtype != torch.complex64:
        raise RuntimeError("state must be complex64")
    if not state.is_contiguous():
        raise RuntimeError("state must be contiguous")
    n = state.numel()
    if n < 2 or n & (n - 1):
        raise RuntimeError("state size must be a power of two >= 2")
    return n.bit_length() - 1


def empty_state(n_qubits: int, device="cuda") -> torch.Tensor:
    return torch.empty(1 << n_qubits, dtype=torch.complex64, device=device)


def state_init(n_qubits: int, device="cuda") -> torch.Tensor:
    s = empty_state(n_qubits, device)
    _h(s.device.index).call("qs_state_init", _ptr(s), int(n_qubits))
    return s


class Plan:
    """A planned circuit (host FP64 fusion + tile passes) resident on the GPU."""

    def __init__(self, n_qubits: int, ops: np.ndarray, device: int | None = None):
        self.n = int(n_qubits)
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.ops, p = _ops_ptr(ops)
        self._h = _h(self.device)
        self.L = self._h.L
        out = C.c_void_p()
        self._h.call("qs_plan_create", self.n, p, int(len(self.ops)), C.byref(out))
        self.ptr = out
        self.info = self.refresh_info()

    def refresh_info(self) -> dict:
        """Planner statistics; n_jit_passes is set at the first execution."""
        info = QsPlanInfo()
        _lib.check(self.L.qs_plan_info_get(self.ptr, C.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in QsPlanInfo._fields_}
        return self.info

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                _wait_uses(self)
                self.L.qs_plan_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def execute(self, state: torch.Tensor) -> torch.Tensor:
        if check_state(state) != self.n:
            raise RuntimeError("state width does not match the plan")
        _h(self.device).call("qs_plan_execute", self.ptr, _ptr(state))
        _record_use(self)
        return state

    def execute_from_zero(self, state: torch.Tensor) -> torch.Tensor:
        if check_state(state) != self.n:
            raise RuntimeError("state width does not match the plan")
        _h(self.device).call("qs_plan_execute_from_zero", self.ptr, _ptr(state))
        _record_use(self)
        return state


class BatchPlan:
    """Many circuits of uneven width, states packed back to back."""

    def __init__(self, widths, op_offsets, ops, state_offsets, device: int | None = None):
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.widths = np.ascontiguousarray(widths, dtype=np.int32)
        self.op_offsets = np.ascontiguousarray(op_offsets, dtype=np.int64)
        self.state_offsets = np.ascontiguousarray(state_offsets, dtype=np.int64)
        self.ops, p = _ops_ptr(ops)
        self.n_amps = int((self.state_offsets + (1 << self.widths.astype(np.int64))).max()) if len(self.widths) else 0
        h = _h(self.device)
        self.L = h.L
        out = C.c_void_p()
        h.call("qs_batch_plan_create", int(len(self.widths)),
               self.widths.ctypes.data_as(C.POINTER(C.c_int32)),
               self.op_offsets.ctypes.data_as(C.POINTER(C.c_int64)), p,
               self.state_offsets.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(out))
        self.ptr = out
        info = QsBatchInfo()
        _lib.check(self.L.qs_batch_plan_info_get(self.ptr, C.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in QsBatchInfo._fields_}

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                _wait_uses(self)
                self.L.qs_batch_plan_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def alloc_states(self) -> torch.Tensor:
        return torch.empty(max(self.n_amps, 2), dtype=torch.complex64, device=f"cuda:{self.device}")

    def execute(self, states: torch.Tensor) -> torch.Tensor:
        if states.numel() < self.n_amps or states.dtype != torch.complex64 or not states.is_cuda:
            raise RuntimeError("states buffer too small or not complex64 CUDA")
        _h(self.device).call("qs_batch_plan_execute", self.ptr, _ptr(states))
        _record_use(self)
        return states


def batch_run(widths, op_offsets, ops, state_offsets, states: torch.Tensor) -> torch.Tensor:
    """One-shot batch (qs_batch_run): every circuit from |0..0> into its
    slice of `states`, planned, run and freed in one call that returns when
    the states are final.  Large batches are planned in slices that overlap
    the GPU running the previous slice."""
    widths = np.ascontiguousarray(widths, dtype=np.int32)
    op_offsets = np.ascontiguousarray(op_offsets, dtype=np.int64)
    state_offsets = np.ascontiguousarray(state_offsets, dtype=np.int64)
    if len(op_offsets) != len(widths) + 1 or len(state_offsets) != len(widths):
        raise ValueError("op_offsets needs n_circuits + 1 entries, state_offsets n_circuits")
    need = int((state_offsets + (1 << widths.astype(np.int64))).max()) if len(widths) else 0
    if states.numel() < need or states.dtype != torch.complex64 or not states.is_cuda:
        raise RuntimeError("states buffer too small or not complex64 CUDA")
    ops, p = _ops_ptr(ops)
    _h(states.device.index).call("qs_batch_run", int(len(widths)), widths.ctypes.data_as(C.POINTER(C.c_int32)),
                                 op_offsets.ctypes.data_as(C.POINTER(C.c_int64)), p, _ptr(states),
                                 state_offsets.ctypes.data_as(C.POINTER(C.c_int64)))
    return states


def run_ops(state: torch.Tensor, ops: np.ndarray) -> torch.Tensor:
    n = check_state(state)
    ops, p = _ops_ptr(ops)
    _h(state.device.index).call("qs_run_circuit", _ptr(state), n, p, int(len(ops)))
    return state


def norm2(state: torch.Tensor) -> float:
    n = check_state(state)
    out = C.c_double()
    _h(state.device.index).call("qs_norm2", _ptr(state), n, C.byref(out))
    return out.value


def renormalize(state: torch.Tensor) -> torch.Tensor:
    n = check_state(state)
    _h(state.device.index).call("qs_renorm", _ptr(state), n)
    return state


def probs(state: torch.Tensor) -> torch.Tensor:
    n = check_state(state)
    out = torch.empty(1 << n, dtype=torch.float32, device=state.device)
    _h(state.device.index).call("qs_probs", _ptr(state), n, _ptr(out))
    return out


def probs_n(states: torch.Tensor, n_amps: int) -> torch.Tensor:
    """|a|^2 of the first n_amps amplitudes of a packed buffer."""
    if states.dtype != torch.complex64 or not states.is_cuda or states.numel() < n_amps or n_amps % 2:
        raise RuntimeError("states must be complex64 CUDA with at least n_amps (even) amplitudes")
    out = torch.empty(int(n_amps), dtype=torch.float32, device=states.device)
    _h(states.device.index).call("qs_probs_n", _ptr(states), int(n_amps), _ptr(out))
    return out


def measure(state: torch.Tensor, target: int, u: float) -> int:
    n = check_state(state)
    F = _lib.fast()
    if F is not None:
        dev = state.get_device()
        return F.measure(_hptr(dev), state.data_ptr(), n, int(target), float(u))
    out = C.c_int()
    _h(state.device.index).call("qs_measure", _ptr(state), n, int(target), float(u), C.byref(out))
    return int(out.value)


def sample_u(state: torch.Tensor, u: torch.Tensor) -> torch.Tensor:
    """Shots for given uniforms u (float64 CUDA): smallest i with cdf[i] >= u."""
    n = check_state(state)
    if u.dtype != torch.float64 or not u.is_cuda or not u.is_contiguous():
        raise RuntimeError("u must be a contiguous float64 CUDA tensor")
    out = torch.empty(u.numel(), dtype=torch.int64, device=state.device)
    F = _lib.fast()
    if F is not None and u.device == state.device:
        F.sample(_hptr(state.get_device()), state.data_ptr(), n, u.data_ptr(), int(u.numel()), out.data_ptr())
        return out
    _h(state.device.index).call("qs_sample", _ptr(state), n, _ptr(u), int(u.numel()), _ptr(out))
    return out


def sample(state: torch.Tensor, shots: int, generator: torch.Generator | None = None) -> torch.Tensor:
    u = torch.rand(int(shots), dtype=torch.float64, device=state.device, generator=generator)
    return sample_u(state, u)


_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def counts(shots: torch.Tensor) -> dict:
    """{outcome: count} of int64 shots held on the device (qs_counts: hash
    histogram on the GPU, only the distinct outcomes copied back), in
    ascending outcome order."""
    keys, cnt = counts_arrays(shots)
    return dict(zip(keys.tolist(), cnt.tolist()))


def counts_arrays(shots: torch.Tensor):
    """(distinct outcomes ascending, their counts) as int64 numpy arrays, from
    qs_counts."""
    if not shots.is_cuda or shots.dtype != torch.int64:
        raise RuntimeError("shots must be an int64 CUDA tensor")
    shots = shots.contiguous()
    n = int(shots.numel())
    if n == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    h = _h(shots.device.index)
    cap = min(n, 1 << 16)
    nd = C.c_int64(0)
    while True:
        pairs = np.empty((cap, 2), dtype=np.int64)
        rc = h.L.qs_counts(h.h, _ptr(shots), n, pairs.ctypes.data_as(C.POINTER(C.c_int64)), cap, C.byref(nd))
        if rc == 0:
            break
        if nd.value > cap:          # more distinct outcomes than room: retry with enough
            cap = int(nd.value)
            continue
        _lib.check(rc, h.h)
    pairs = pairs[: nd.value]
    order = np.argsort(pairs[:, 0], kind="stable")
    return pairs[order, 0], pairs[order, 1]


def seed_uniforms(seed: int, count: int) -> np.ndarray:
    """The native server's per-request uniforms: splitmix64 (Steele, Lea and
    Flood, 2014) from `seed`, top 53 bits scaled to [0, 1).  Sampling with
    these gives the same shots as a NativeServer request with that seed."""
    i = np.arange(1, int(count) + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(int(seed) & (2 ** 64 - 1)) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z ^= z >> np.uint64(31)
    return (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def sample_batched(states: torch.Tensor, widths, offsets, shots, seeds) -> torch.Tensor:
    """Shots of many states (any widths) packed in one complex64 CUDA tensor,
    in three launches: state t has widths[t] qubits from amplitude offsets[t]
    and gets shots[t] shots drawn with seed_uniforms(seeds[t], shots[t]) (the
    same shots as sample_seeded).  Returns one int64 device tensor, the
    states' shots in order."""
    if states.dtype != torch.complex64 or not states.is_cuda or not states.is_contiguous():
        raise RuntimeError("states must be a contiguous complex64 CUDA tensor")
    w = np.ascontiguousarray(widths, dtype=np.int32)
    o = np.ascontiguousarray(offsets, dtype=np.int64)
    k = np.ascontiguousarray(shots, dtype=np.int64)
    sd = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64))
    if not (w.shape == o.shape == k.shape == sd.shape) or w.ndim != 1:
        raise ValueError("widths, offsets, shots and seeds need one entry per state")
    if len(w) and int((o + (np.int64(1) << w.astype(np.int64))).max()) > states.numel():
        raise ValueError("a state runs past the end of the states tensor")
    out = torch.empty(int(k.sum()), dtype=torch.int64, device=states.device)
    _h(states.device.index).call("qs_sample_batched", _ptr(states), int(len(w)),
                                 w.ctypes.data_as(C.POINTER(C.c_int32)), o.ctypes.data_as(C.POINTER(C.c_int64)),
                                 k.ctypes.data_as(C.POINTER(C.c_int64)), sd.ctypes.data_as(C.POINTER(C.c_uint64)),
                                 _ptr(out) if out.numel() else None)
    return out


def sample_seeded(state: torch.Tensor, shots: int, seed: int) -> torch.Tensor:
    """Shots drawn with seed_uniforms(seed, shots) (device tensor)."""
    u = torch.from_numpy(seed_uniforms(seed, shots)).to(state.device, non_blocking=False)
    return sample_u(state, u)


def _masks(ps):
    x = np.ascontiguousarray(ps.x, dtype=np.uint64)
    z = np.ascontiguousarray(ps.z, dtype=np.uint64)
    c = np.ascontiguousarray(ps.real_coefs(), dtype=np.float64)
    return x, z, c


def expect_pauli_sum(state: torch.Tensor, ps) -> float:
    n = check_state(state)
    x, z, c = _masks(ps)
    out = C.c_double()
    _h(state.device.index).call("qs_expect_pauli_sum", _ptr(state), n,
                                x.ctypes.data_as(C.POINTER(C.c_uint64)), z.ctypes.data_as(C.POINTER(C.c_uint64)),
                                c.ctypes.data_as(C.POINTER(C.c_double)), int(len(c)), C.byref(out))
    return out.value


def apply_pauli_sum(state: torch.Tensor, ps) -> torch.Tensor:
    n = check_state(state)
    x, z, c = _masks(ps)
    out = torch.empty_like(state)
    _h(state.device.index).call("qs_apply_pauli_sum", _ptr(state), _ptr(out), n,
                                x.ctypes.data_as(C.POINTER(C.c_uint64)), z.ctypes.data_as(C.POINTER(C.c_uint64)),
                                c.ctypes.data_as(C.POINTER(C.c_double)), int(len(c)))
    return out


def adjoint_gradient(n: int, ops: np.ndarray, n_params: int, params: np.ndarray, ps, device: int | None = None):
    """Energies [B] and gradients [B, n_params] (FP64) for parameter vectors
    params [B, n_params]."""
    dev = torch.cuda.current_device() if device is None else int(device)
    params = np.ascontiguousarray(params, dtype=np.float64).reshape(-1, n_params) if n_params else \
        np.zeros((int(params.shape[0]) if params.ndim else 1, 0))
    B = params.shape[0]
    ops, p = _ops_ptr(ops)
    x, z, c = _masks(ps)
    work = torch.empty(B * 3 * (1 << n), dtype=torch.complex64, device=f"cuda:{dev}")
    e = np.zeros(B, dtype=np.float64)
    g = np.zeros((B, max(n_params, 1)), dtype=np.float64)
    _h(dev).call("qs_adjoint_gradient", int(n), p, int(len(ops)), int(n_params),
                 params.ctypes.data_as(C.POINTER(C.c_double)), int(B),
                 x.ctypes.data_as(C.POINTER(C.c_uint64)), z.ctypes.data_as(C.POINTER(C.c_uint64)),
                 c.ctypes.data_as(C.POINTER(C.c_double)), int(len(c)), _ptr(work),
                 e.ctypes.data_as(C.POINTER(C.c_double)), g.ctypes.data_as(C.POINTER(C.c_double)))
    return e, g[:, :n_params]


def launch_count(device: int | None = None) -> int:
    return _h(device).launches()
