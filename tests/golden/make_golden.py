"""Generate golden fixtures from the reference's own Python code.

Run with QSIM_REFERENCE set to the root of a checkout of the reference
project (read-only is enough), e.g.
``QSIM_REFERENCE=<path to the reference> python tests/golden/make_golden.py``.
Writes tests/golden/*.npz, so the tests themselves never need the reference
tree.

Pieces of the reference that run on a CPU without qiskit and without its
compiled extension:
  * bwk/python/blackwell_kernels/qv8.py   generate_qv8_circuits, qv8_simulate_ref (torch, CPU)
  * bwk/python/blackwell_kernels/qv4.py   generate_qv4_circuits, qv4_simulate_numpy
    (its module-level `import blackwell_kernels._C` is satisfied by an empty
    stub module; only the pure-Python functions are called)
  * blackwell_backend/chebyshev.py        chebyshev_coefficients (scipy.special.jv)
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

import numpy as np

REF = os.environ.get("QSIM_REFERENCE", "")
OUT = os.path.dirname(os.path.abspath(__file__))


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def qv8():
    m = _load("ref_qv8", os.path.join(REF, "bwk/python/blackwell_kernels/qv8.py"))
    gm, gq, G = m.generate_qv8_circuits(6, seed=42)
    probs = m.qv8_simulate_ref(gm.double().float(), gq, 6)
    np.savez_compressed(os.path.join(OUT, "qv8_ref.npz"), gate_matrices=gm.numpy(), gate_qubits=gq.numpy(),
                        probs=probs.numpy(), G=G)


def qv4():
    pkg = types.ModuleType("blackwell_kernels")
    pkg.__path__ = []
    sys.modules.setdefault("blackwell_kernels", pkg)
    sys.modules.setdefault("blackwell_kernels._C", types.ModuleType("blackwell_kernels._C"))
    m = _load("ref_qv4", os.path.join(REF, "bwk/python/blackwell_kernels/qv4.py"))
    gd, pid = m.generate_qv4_circuits(12, rng=np.random.default_rng(7))
    probs = m.qv4_simulate_numpy(gd, pid)
    hop = m.heavy_output_probability(probs)
    np.savez_compressed(os.path.join(OUT, "qv4_ref.npz"), gate_data=gd, pair_ids=pid, probs=probs, hop=hop)


def cheb():
    m = _load("ref_cheb", os.path.join(REF, "blackwell_backend/chebyshev.py"))
    cases = [(1.0, 4.0, 1e-10), (0.5, 10.0, 1e-12), (-2.0, 3.5, 1e-8), (5.0, 64.0, 1e-6), (10.0, 32.0, 1e-6),
             (0.01, 1.0, 1e-10)]
    rows = {}
    for i, (t, b, p) in enumerate(cases):
        c, K, tail = m.chebyshev_coefficients(t, b, p)
        rows[f"c{i}"] = c
        rows[f"meta{i}"] = np.array([t, b, p, K, tail])
    np.savez_compressed(os.path.join(OUT, "cheb_coeffs_ref.npz"), n=len(cases), **rows)


if __name__ == "__main__":
    if not REF or not os.path.isdir(REF):
        sys.exit("set QSIM_REFERENCE to the root of a checkout of the reference project")
    qv8()
    qv4()
    cheb()
    print("golden fixtures written to", OUT)
