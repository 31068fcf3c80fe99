"""The C-ABI library loads and exports every symbol include/qsim.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "qsim.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qs_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    import __graft_entry__  # noqa: F401  (puts the package on sys.path)
    from qsim_b200 import _lib
    if not os.path.exists(_lib.lib_path()):
        import importlib
        ge = importlib.import_module("__graft_entry__")
        ge.build()
    return ctypes.CDLL(_lib.lib_path())


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("qs_create", "qs_apply_1q", "qs_apply_2q", "qs_plan_create", "qs_sample", "qs_cheb_evolve",
                 "qs_batch_run", "qs_adjoint_gradient", "qs_expect_pauli_sum"):
        assert must in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"missing exports: {missing}"


def test_ctypes_signatures_cover_header():
    from qsim_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.SIGNATURES), set(declared_symbols()) - set(_lib.SIGNATURES)


def test_version_and_null_handle_errors(lib):
    lib.qs_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.qs_version()
    lib.qs_last_error.restype = ctypes.c_char_p
    # calls with a null handle fail cleanly (no GPU needed)
    assert lib.qs_sync(None) == 1
    assert b"null handle" in lib.qs_last_error(None)


def test_fast_extension_binds_the_same_library():
    """blackwell_kernels' per-gate calls go through the _qsfast extension (no
    ctypes marshalling); it links the in-tree libqsim.so and reports errors
    as QsimError."""
    import pytest
    from qsim_b200 import _lib
    F = _lib.fast()
    assert F is not None
    with pytest.raises(_lib.QsimError, match="null handle"):
        F.apply_1q_dev(0, 0, 3, 0, 0)
    with pytest.raises(RuntimeError, match="0-7"):
        F.apply_mc1q_dev(0, 0, 3, 0, list(range(8)), 0)
    # every call the Python layer routes through the extension, each
    # reaching the library (a null handle is refused before any CUDA call)
    for name, args in [("apply_2q_dev", (0, 0, 3, 0, 0, 1)), ("apply_gates_fused_dev", (0, 0, 3, 0, 0, 2)),
                       ("apply_diag1_dev", (0, 0, 3, 0, 0)), ("apply_diag2_dev", (0, 0, 3, 0, 0, 1)),
                       ("apply_phase", (0, 0, 3, 1.0, 0.0, 0)), ("apply_mc2q_dev", (0, 0, 3, 0, [2], 0, 1)),
                       ("measure", (0, 0, 3, 0, 0.5)), ("sample", (0, 0, 3, 0, 10, 0))]:
        with pytest.raises(_lib.QsimError, match="null handle"):
            getattr(F, name)(*args)
    with pytest.raises(TypeError, match="expected 5 arguments"):
        F.measure(0, 0, 3, 0)


def test_autotune_table_set_get_and_range(lib):
    """A tuned entry set by hand reads back through qs_autotune_get (host-side
    table, no GPU work); entries outside the kernels' shapes are rejected."""
    lib.qs_autotune_set.argtypes = [ctypes.c_int] * 4
    lib.qs_autotune_get.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_int)]
    dev = 7  # a device index no GPU test uses
    assert lib.qs_autotune_set(dev, 17, 13, 5) == 0
    tb, bb = ctypes.c_int(0), ctypes.c_int(0)
    assert lib.qs_autotune_get(dev, 17, ctypes.byref(tb), ctypes.byref(bb)) == 0
    assert (tb.value, bb.value) == (13, 5)
    for bad in ((dev, 17, 9, 5), (dev, 17, 15, 5), (dev, 17, 13, 1), (dev, 17, 13, 6), (-1, 17, 13, 5),
                (dev, 0, 13, 5)):
        assert lib.qs_autotune_set(*bad) != 0
    assert lib.qs_autotune_get(dev, 17, ctypes.byref(tb), ctypes.byref(bb)) == 0
    assert (tb.value, bb.value) == (13, 5)
    assert lib.qs_autotune_clear(dev) == 0
    assert lib.qs_autotune_get(dev, 17, ctypes.byref(tb), ctypes.byref(bb)) != 0
