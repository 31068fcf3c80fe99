"""Build libqsim.so (sm_100a) in-tree.

Every translation unit under csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo`` (no --use_fast_math: the
compensated arithmetic relies on IEEE rounding) and linked into
``lib/libqsim.so`` with the CUDA runtime linked statically.  Object files go to
``_build/``.  Run ``python build_lib.py`` or call :func:`build`.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libqsim.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", INCLUDE, "-I", CSRC]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _deps() -> list[str]:
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + [
        os.path.join(INCLUDE, "qsim.h")]


def _compile(nvcc: str, src: str, obj: str, verbose: bool, extra: list[str]) -> None:
    lang = ["-x", "cu"] if src.endswith(".cu") else []
    cmd = [nvcc, *lang, *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile csrc/ into lib/libqsim.so; returns the library path."""
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = _sources()
    dep_mtime = max(os.path.getmtime(d) for d in _deps())
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or ptxas_info or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), dep_mtime):
            jobs.append((s, o))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = [ex.submit(_compile, nvcc, s, o, verbose or ptxas_info, extra) for s, o in jobs]
            for f in futs:
                f.result()
    if jobs or not os.path.exists(LIB):
        cmd = [nvcc, *ARCH, "-shared", "-Xlinker", "-soname=libqsim.so", "-o", LIB, *objs, "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


PYEXT_SRC = os.path.join(HERE, "pyext", "qs_fast.c")


def pyext_path() -> str:
    import sysconfig
    return os.path.join(LIBDIR, "_qsfast" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def build_pyext(force: bool = False) -> str | None:
    """The CPython extension behind blackwell_kernels' per-gate calls
    (pyext/qs_fast.c, linked against lib/libqsim.so).  Returns its path, or
    None when no C compiler or Python headers are available (the ctypes path
    is used then)."""
    import sysconfig
    out = pyext_path()
    inc = sysconfig.get_paths().get("include", "")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(PYEXT_SRC),
                                                                           os.path.getmtime(LIB)):
        return out
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc or not os.path.exists(os.path.join(inc, "Python.h")):
        return None
    cmd = [cc, "-O2", "-shared", "-fPIC", "-I", inc, PYEXT_SRC, "-L", LIBDIR, "-lqsim",
           "-Wl,-rpath,$ORIGIN", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"extension build failed:\n{r.stdout}\n{r.stderr}")
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    build_pyext()
    print(LIB)
