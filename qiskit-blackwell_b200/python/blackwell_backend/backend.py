"""A Qiskit BackendV2-shaped backend over libqsim.

Qiskit's ``BackendV2`` base class needs qiskit itself, which this package
does not depend on; ``BlackwellBackend`` has the same shape, so code written
against a BackendV2 (``backend.target``, ``backend.options``,
``backend.run(circuits, shots=...)`` returning a job whose ``result()`` is a
``Result``) works unchanged:

    backend = BlackwellBackend()
    job = backend.run([qc1, qc2], shots=2048, seed_simulator=7)
    counts = job.result().get_counts(1)

Circuits go through ``HybridSimulator``'s routing (a list of small circuits
runs as one batch plan, large ones on the plain plan path); counts are
histogrammed on the device.  The reference exposes only
``BlackwellSimulator.run`` (blackwell_backend/simulator.py:555-604); each
experiment of the result here has that call's shape (hex counts, header
{name, n_qubits}, shots).
"""
from __future__ import annotations

import itertools
import time
import uuid

from qsim_b200.circuit import LOWERABLE

from .hybrid import HybridSimulator
from .simulator import Result

MAX_QUBITS = 34  # QS_MAX_QUBITS of include/qsim.h


class Options:
    """Run options (BackendV2.options): shots and seed_simulator."""

    def __init__(self, **kw):
        self.shots = 1024
        self.seed_simulator = None
        self.update_options(**kw)

    def update_options(self, **kw):
        for k, v in kw.items():
            if k not in ("shots", "seed_simulator"):
                raise AttributeError(f"unknown option {k!r}")
            setattr(self, k, v)

    def get(self, k, default=None):
        return getattr(self, k, default)


class Target:
    """The subset of qiskit.transpiler.Target a caller inspects: the qubit
    count and the operations the backend runs without transpilation (any
    other gate with a matrix, a controlled base gate or a definition is
    lowered as well, see qsim_b200.circuit._convert)."""

    def __init__(self, num_qubits: int):
        self.num_qubits = num_qubits
        self.operation_names = sorted(LOWERABLE - {"mcu"})

    def instruction_supported(self, operation_name: str, qargs=None) -> bool:
        if operation_name not in self.operation_names:
            return False
        return qargs is None or all(0 <= int(q) < self.num_qubits for q in qargs)

    def __contains__(self, name):
        return name in self.operation_names


class BlackwellJob:
    """JobV1-shaped: job_id(), status(), done(), result()."""

    def __init__(self, backend, job_id: str, results, time_taken: float):
        self._backend, self._id, self._results, self._t = backend, job_id, results, time_taken

    def job_id(self) -> str:
        return self._id

    def backend(self):
        return self._backend

    def status(self) -> str:
        return "DONE"

    def done(self) -> bool:
        return True

    def result(self, timeout=None) -> Result:
        exps = [r.results[0] for r in self._results]
        return Result("blackwell_simulator", self._backend.backend_version, "", self._id,
                      all(r.success for r in self._results), exps, self._t)


class BlackwellBackend:
    name = "blackwell_simulator"
    description = "complex64 statevector simulator on B200 (libqsim, sm_100a)"
    backend_version = "0.1.0"
    _ids = itertools.count()

    def __init__(self, device="cuda", kernel_path=None, **options):
        self._hybrid = HybridSimulator(kernel_path=kernel_path, device=device)
        self._options = Options(**options)
        self._target = Target(MAX_QUBITS)

    @property
    def target(self) -> Target:
        return self._target

    @property
    def num_qubits(self) -> int:
        return self._target.num_qubits

    @property
    def operation_names(self):
        return self._target.operation_names

    @property
    def options(self) -> Options:
        return self._options

    @property
    def max_circuits(self):
        return None

    def set_options(self, **kw):
        self._options.update_options(**kw)

    def run(self, run_input, **options) -> BlackwellJob:
        """Runs one circuit or a list; options override shots and
        seed_simulator for this call.  Circuit k of a list samples with
        seed_simulator + k."""
        opts = Options(shots=self._options.shots, seed_simulator=self._options.seed_simulator)
        opts.update_options(**options)
        circuits = list(run_input) if isinstance(run_input, (list, tuple)) else [run_input]
        t0 = time.perf_counter()
        results = self._hybrid.run(circuits, shots=int(opts.shots), seed=opts.seed_simulator)
        return BlackwellJob(self, f"blackwell-{next(self._ids)}-{uuid.uuid4().hex[:8]}", results,
                            time.perf_counter() - t0)

    def close(self):
        self._hybrid.close()
