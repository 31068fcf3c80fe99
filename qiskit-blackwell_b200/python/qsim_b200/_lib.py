"""ctypes binding of libqsim.so (the C ABI declared in include/qsim.h).

The library is located next to this package (``../../lib/libqsim.so``) unless
``QSIM_LIB`` names another build (the A/B hook that mirrors the reference's
``kernel_path`` / ``BLACKWELL_KERNEL_PATH``, blackwell_backend/simulator.py:43-63).
There is no fallback: if the library or a GPU is missing, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.normpath(os.path.join(_HERE, "..", "..", "lib", "libqsim.so"))

QS_OK = 0
QS_ERR_INVALID = 1
QS_ERR_CUDA = 2
QS_ERR_NOMEM = 3
QS_ERR_TIMEOUT = 4
QS_ERR_BUDGET = 5

# op kinds (include/qsim.h)
OP_U1, OP_U2, OP_DIAG1, OP_DIAG2, OP_MCU1, OP_MCU2, OP_MCX, OP_MCSWAP, OP_MCPHASE, OP_Y, OP_RX, OP_RY, OP_RZ = range(1, 14)
OP_DEPOLARIZE, OP_AMP_DAMP, OP_DEPHASE = 20, 21, 22


class QsOp(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nq", C.c_int32), ("q", C.c_int32 * 8), ("param", C.c_int32),
                ("flags", C.c_int32), ("m", C.c_double * 32)]


class QsPlanInfo(C.Structure):
    _fields_ = [("n_qubits", C.c_int32), ("tile_bits", C.c_int32), ("n_passes", C.c_int32),
                ("n_blocks", C.c_int32), ("n_ops_in", C.c_int64), ("n_ops_fused", C.c_int64),
                ("bytes_moved", C.c_double), ("flops", C.c_double), ("n_device_ops", C.c_int64),
                ("n_jit_passes", C.c_int32), ("reserved", C.c_int32)]


class QsBatchInfo(C.Structure):
    _fields_ = [("n_circuits", C.c_int32), ("n_launches", C.c_int32), ("n_items", C.c_int64),
                ("max_passes", C.c_int32), ("n_tc_launches", C.c_int32), ("bytes_moved", C.c_double), ("flops", C.c_double)]


class QsServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("queued", C.c_int64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("throughput_rps", C.c_double),
                ("budget_bytes", C.c_int64), ("free_bytes", C.c_int64)]


class QsimError(RuntimeError):
    """Raised when a libqsim call returns a non-zero status (the reference
    raises RuntimeError from TORCH_CHECK for the same conditions)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"qsim error {code}: {msg}")
        self.code = code


_vp = C.c_void_p
_i = C.c_int
_i64 = C.c_int64
_u64 = C.c_uint64
_d = C.c_double
_f = C.c_float
_pf = C.POINTER(C.c_float)
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)
_pi32 = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)
_pu64 = C.POINTER(C.c_uint64)
_pop = C.POINTER(QsOp)

# name -> (restype, argtypes)
SIGNATURES = {
    "qs_create": (_i, [_i, C.POINTER(_vp)]),
    "qs_destroy": (_i, [_vp]),
    "qs_set_stream": (_i, [_vp, _vp]),
    "qs_get_stream": (_vp, [_vp]),
    "qs_sync": (_i, [_vp]),
    "qs_last_error": (C.c_char_p, [_vp]),
    "qs_version": (C.c_char_p, []),
    "qs_set_tile_bits": (_i, [_vp, _i]),
    "qs_set_block_bits": (_i, [_vp, _i]),
    "qs_set_jit": (_i, [_vp, _i, _i]),
    "qs_launch_count": (_i64, [_vp]),
    "qs_counts": (_i, [_vp, _vp, _i64, _pi64, _i64, _pi64]),
    "qs_device_status": (_i, [_vp, _pi]),
    "qs_set_wait_test": (_i, [_vp, _i]),
    "qs_set_batch_queue": (_i, [_vp, _i]),
    "qs_set_tensor_cores": (_i, [_vp, _i]),
    "qs_state_init": (_i, [_vp, _vp, _i]),
    "qs_state_alloc": (_i, [_vp, _i, C.POINTER(C.c_void_p)]),
    "qs_state_free": (_i, [_vp, _vp]),
    "qs_state_copy_to_host": (_i, [_vp, _vp, _i, _vp]),
    "qs_state_copy_from_host": (_i, [_vp, _vp, _i, _vp]),
    "qs_state_init_basis": (_i, [_vp, _vp, _i, _u64]),
    "qs_state_init_batched": (_i, [_vp, _vp, _i, _i]),
    "qs_apply_1q": (_i, [_vp, _vp, _i, _pf, _i]),
    "qs_apply_2q": (_i, [_vp, _vp, _i, _pf, _i, _i]),
    "qs_apply_diag1": (_i, [_vp, _vp, _i, _pf, _i]),
    "qs_apply_phase": (_i, [_vp, _vp, _i, _f, _f, _i]),
    "qs_apply_diag2": (_i, [_vp, _vp, _i, _pf, _i, _i]),
    "qs_apply_1q_dev": (_i, [_vp, _vp, _i, _vp, _i]),
    "qs_apply_gates_fused_dev": (_i, [_vp, _vp, _i, _vp, _vp, _i]),
    "qs_apply_2q_dev": (_i, [_vp, _vp, _i, _vp, _i, _i]),
    "qs_apply_diag1_dev": (_i, [_vp, _vp, _i, _vp, _i]),
    "qs_apply_mc1q_dev": (_i, [_vp, _vp, _i, _vp, _pi, _i, _i]),
    "qs_apply_diag2_dev": (_i, [_vp, _vp, _i, _vp, _i, _i]),
    "qs_apply_mc2q_dev": (_i, [_vp, _vp, _i, _vp, _pi, _i, _i, _i]),
    "qs_apply_mc1q": (_i, [_vp, _vp, _i, _pf, _pi, _i, _i]),
    "qs_apply_mc2q": (_i, [_vp, _vp, _i, _pf, _pi, _i, _i, _i]),
    "qs_apply_mcx": (_i, [_vp, _vp, _i, _pi, _i, _i]),
    "qs_apply_mcswap": (_i, [_vp, _vp, _i, _pi, _i, _i, _i]),
    "qs_apply_mcz": (_i, [_vp, _vp, _i, _pi, _i]),
    "qs_apply_gates_fused": (_i, [_vp, _vp, _i, _pf, _pi, _i]),
    "qs_apply_1q_batched": (_i, [_vp, _vp, _i, _i, _pf, _i]),
    "qs_apply_gates_batched_fused": (_i, [_vp, _vp, _i, _i, _pf, _pi, _i]),
    "qs_plan_create": (_i, [_vp, _i, _pop, _i, C.POINTER(_vp)]),
    "qs_plan_info_get": (_i, [_vp, C.POINTER(QsPlanInfo)]),
    "qs_plan_execute": (_i, [_vp, _vp, _vp]),
    "qs_plan_execute_from_zero": (_i, [_vp, _vp, _vp]),
    "qs_plan_destroy": (_i, [_vp]),
    "qs_plan_analyze": (_i, [_i, _pop, _i, _i, C.POINTER(QsPlanInfo)]),
    "qs_plan_jit_check": (_i, [_i, _pop, _i, _i, _i, C.POINTER(C.c_int)]),
    "qs_autotune_batch": (_i, [_vp, _i, _vp, _vp, _pop]),
    "qs_autotune_get": (_i, [_i, _i, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "qs_autotune_set": (_i, [_i, _i, _i, _i]),
    "qs_autotune_clear": (_i, [_i]),
    "qs_server_create": (_i, [_i, C.c_int64, _i, C.POINTER(C.c_void_p)]),
    "qs_server_destroy": (_i, [_vp]),
    "qs_server_submit_circuit": (_i, [_vp, _i, _pop, _i, C.c_int64, C.c_uint64, _d, C.POINTER(C.c_int64)]),
    "qs_server_submit_gradient": (_i, [_vp, _i, _pop, _i, _i, _vp, _i, _vp, _vp, _vp, _i, _d,
                                       C.POINTER(C.c_int64)]),
    "qs_server_submit_evolution": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _i, _vp, _i, _d, _d, C.POINTER(C.c_int64)]),
    "qs_server_wait": (_i, [_vp, C.c_int64, _d, C.POINTER(C.c_int)]),
    "qs_server_cancel": (_i, [_vp, C.c_int64]),
    "qs_server_request_error": (C.c_char_p, [_vp, C.c_int64]),
    "qs_server_result_samples": (_i, [_vp, C.c_int64, _vp, C.c_int64]),
    "qs_server_result_gradient": (_i, [_vp, C.c_int64, _vp, _vp]),
    "qs_server_result_state": (_i, [_vp, C.c_int64, _vp]),
    "qs_server_release": (_i, [_vp, C.c_int64]),
    "qs_server_stats_get": (_i, [_vp, C.POINTER(QsServerStats)]),
    "qs_plan_program": (_i, [_i, _pop, _i, _i, _i, _i, _vp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "qs_run_circuit": (_i, [_vp, _vp, _i, _pop, _i]),
    "qs_norm2": (_i, [_vp, _vp, _i, _pd]),
    "qs_renorm": (_i, [_vp, _vp, _i]),
    "qs_probs": (_i, [_vp, _vp, _i, _vp]),
    "qs_probs_n": (_i, [_vp, _vp, _i64, _vp]),
    "qs_measure": (_i, [_vp, _vp, _i, _i, _d, _pi]),
    "qs_sample": (_i, [_vp, _vp, _i, _vp, _i64, _vp]),
    "qs_expect_z": (_i, [_vp, _vp, _i, _u64, _pd]),
    "qs_expect_pauli_sum": (_i, [_vp, _vp, _i, _pu64, _pu64, _pd, _i, _pd]),
    "qs_expect_pauli_sum_noalloc": (_i, [_vp, _vp, _i, _pu64, _pu64, _pd, _i, _pd]),
    "qs_spmv_csr": (_i, [_vp, _vp, _vp, _vp, _i64, _vp, _vp, _d, _d, _d, _d]),
    "qs_cheb_step": (_i, [_vp, _vp, _vp, _vp, _i64]),
    "qs_cheb_accum": (_i, [_vp, _vp, _vp, _d, _d, _i64]),
    "qs_cheb_step_accum": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _d, _i64]),
    "qs_cheb_evolve": (_i, [_vp, _vp, _vp, _vp, _i, _vp, _vp, _pd, _i, _d, _vp]),
    "qs_cheb_evolve_pauli": (_i, [_vp, _i, _vp, _vp, _pu64, _pu64, _pd, _i, _pd, _i, _d, _vp]),
    "qs_apply_depolarizing": (_i, [_vp, _vp, _i, _i, _d, _d, _pi32]),
    "qs_apply_amplitude_damping": (_i, [_vp, _vp, _i, _i, _d, _d, _pi32]),
    "qs_apply_dephasing": (_i, [_vp, _vp, _i, _i, _d, _d, _pi32]),
    "qs_sample_batched": (_i, [_vp, _vp, _i, _pi32, _pi64, _pi64, _pu64, _vp]),
    "qs_noise_program": (_i, [_i, _pop, _i, _i, _vp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "qs_noise_trajectories": (_i, [_vp, _i, _pop, _i, _i, _pu64, _vp, C.POINTER(C.c_uint8)]),
    "qs_batch_run": (_i, [_vp, _i, _pi32, _pi64, _pop, _vp, _pi64]),
    "qs_batch_plan_create": (_i, [_vp, _i, _pi32, _pi64, _pop, _pi64, C.POINTER(_vp)]),
    "qs_batch_plan_execute": (_i, [_vp, _vp, _vp]),
    "qs_batch_plan_info_get": (_i, [_vp, C.POINTER(QsBatchInfo)]),
    "qs_batch_plan_destroy": (_i, [_vp]),
    "qs_adjoint_gradient": (_i, [_vp, _i, _pop, _i, _i, _pd, _i, _pu64, _pu64, _pd, _i, _vp, _pd, _pd]),
    "qs_apply_pauli_sum": (_i, [_vp, _vp, _vp, _i, _pu64, _pu64, _pd, _i]),
}

_lib = None
_lib_lock = threading.Lock()


def lib_path() -> str:
    return os.environ.get("QSIM_LIB", DEFAULT_LIB)


def load(path: str | None = None):
    """Load (once) and return the ctypes library with typed entry points."""
    global _lib
    with _lib_lock:
        if _lib is not None and path is None:
            return _lib
        p = path or lib_path()
        if not os.path.exists(p):
            raise FileNotFoundError(
                f"libqsim.so not found at {p}; build it with `python qiskit-blackwell_b200/build_lib.py`")
        L = C.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if path is None:
            _lib = L
        return L


def check(rc: int, handle=None) -> None:
    if rc != QS_OK:
        L = load()
        msg = L.qs_last_error(handle)
        raise QsimError(rc, msg.decode() if msg else "")


class Handle:
    """Owns one qs_handle_t (streams, scratch) on one device."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        rc = self.L.qs_create(int(device), C.byref(h))
        if rc != QS_OK:
            msg = self.L.qs_last_error(None)
            raise QsimError(rc, msg.decode() if msg else "qs_create failed")
        self.h = h
        self.device = int(device)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.qs_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def call(self, name: str, *args):
        rc = getattr(self.L, name)(self.h, *args)
        if rc != QS_OK:
            msg = self.L.qs_last_error(self.h)
            raise QsimError(rc, msg.decode() if msg else name)
        return rc

    def set_stream(self, stream_ptr: int | None) -> None:
        self.call("qs_set_stream", C.c_void_p(stream_ptr or 0))

    def launches(self) -> int:
        return int(self.L.qs_launch_count(self.h))


_handles = threading.local()

_fast_mod = False   # not looked up yet


def fast():
    """The _qsfast CPython extension (direct calls into the per-gate entry
    points, no ctypes marshalling) when it is built and binds the same
    libqsim.so this process loaded; None otherwise (QSIM_LIB naming another
    build, or no extension)."""
    global _fast_mod
    if _fast_mod is False:
        _fast_mod = None
        try:
            import importlib.machinery
            import importlib.util
            import sysconfig
            lib = load()
            libdir = os.path.dirname(DEFAULT_LIB)
            path = os.path.join(libdir, "_qsfast" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))
            if lib is not None and os.path.exists(path) and os.path.realpath(lib_path()) == os.path.realpath(DEFAULT_LIB):
                loader = importlib.machinery.ExtensionFileLoader("_qsfast", path)
                spec = importlib.util.spec_from_file_location("_qsfast", path, loader=loader)
                mod = importlib.util.module_from_spec(spec)
                loader.exec_module(mod)
                mod.set_error(QsimError)
                _fast_mod = mod
        except Exception:
            _fast_mod = None
    return _fast_mod


def handle(device: int = 0, stream_ptr: int | None = None) -> Handle:
    """Per-thread, per-device handle bound to the given CUDA stream (torch's
    current stream when called from the torch-facing wrappers)."""
    d = getattr(_handles, "d", None)
    if d is None:
        d = _handles.d = {}
    h = d.get(device)
    if h is None:
        h = d[device] = Handle(device)
        h._stream = None
    if stream_ptr is not None and stream_ptr != h._stream:
        h.set_stream(stream_ptr)
        h._stream = stream_ptr
    return h
