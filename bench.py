"""Benchmark driver (one JSON line on rank 0).

Workloads (--workload):
  layers32  (default) 32-qubit state (2^32 complex64 = 32 GiB), 20 layers of
            Haar U(2) on every qubit + CZ brickwork + a Toffoli every 5th
            layer (954 gates).  value = gates/s of the fused tile passes on a
            state resident in HBM; e2e = gates/s of the public call path
            (host op list -> plan upload -> passes -> 1024 shots -> host).
  qv_batch  4096 Quantum-Volume circuits, widths uniform in [10, 20], depth =
            width, per-circuit seeds; value = circuits/s of the batch engine,
            beside one plan per circuit on the same GPU.
  qv12      one 12-qubit, depth-12 QV circuit; value = circuits/s.
  adjoint   20-qubit EfficientSU2 (4 reps, 200 parameters), 256-term
            observable, batch 64; value = gradients/s, with the energy-only
            forward timed for the gradient/forward ratio.
  serving   seeded Poisson request streams (QV circuits with shots, ansatz
            gradients, Chebyshev evolutions) at rates 50..2000 req/s through
            the continuous-batching server; value = served requests/s at the
            highest rate, p50/p99 per rate, serial plain execution beside it.
  chebyshev exp(-iHt)|psi> at 22 qubits (84 Pauli terms, t = 10); value =
            evolutions/s of the matrix-free path, the CSR path beside it.
  noisy     12-qubit noisy brickwork, 8192 seeded trajectories per step;
            value = trajectories/s.
  micro     the reference's published single-operation times at 20 qubits
            and QV-20 end to end with 8192 shots; value = circuits/s.
  qv_plain  one QV circuit (--qubits) on the plain path.

--impl reference times the CPU implementation of the same workload on a
bounded sample, scaled to the metric's unit, with every host core busy: the
FP64 statevector restatement (oracle/sv64.c, OpenMP) for circuits, and for
trajectories and evolutions one worker process per core (numpy trajectories,
scipy expm_multiply).  It is the only other place this file runs oracle/ code
besides the cpu_baseline leg.

Multi-GPU (torchrun, one process per GPU): the workloads do not shard, so
each rank runs an independent replica; value = total units / max-over-ranks
device time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "qiskit-blackwell_b200", "python"), os.path.join(ROOT, "qiskit-blackwell_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

# The headline metric every line reports under.
METRIC = "served circuits/s + p50/p99 vs per-circuit launches at 1\u2212F\u22641e-6; HBM GB/s"


# ------------------------------------------------------------ distributed
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws, backend):
    import datetime
    import torch.distributed as dist
    if ws > 1 and not dist.is_initialized():
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def reduce_max(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return float(x)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed
    region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"]}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def describe(workload: str, args) -> str:
    """The workload named by what it is, with its sizes: the `config`
    string both arms print (no GPU needed)."""
    if workload == "layers32":
        from qsim_b200 import workloads as W
        n = args.qubits
        ngates = len(W.layers_ops(n, 20, seed=0))
        return (f"layers32: {n} qubits (2^{n} complex64 = {(8 << n) >> 30} GiB), 20 layers "
                f"U(2)+CZ brickwork+Toffoli/5, {ngates} gates, seed 0")
    if workload == "qv_batch":
        return f"qv_batch: {args.circuits} QV circuits, widths U[10,20], depth=width, seeds 1e6*1+i"
    if workload == "qv12":
        return "qv12: 12 qubits, depth 12, seed 0 (72 U(4))"
    if workload == "serving":
        return (f"serving: {args.requests} seeded requests (50% QV 10-28q 1024 shots, 25% EfficientSU2 "
                f"energy+gradient 12-22q, 25% Chebyshev evolution 12-22q), Poisson arrivals at "
                f"{args.rates} req/s, the sequence replayed at each rate; 150 GB budget, {args.workers} worker "
                f"streams, {args.server} server")
    if workload == "adjoint":
        n = args.qubits if args.qubits != 32 else 20
        return f"adjoint: EfficientSU2 {n} qubits, 4 reps, {2 * n * 5} params, 256-term observable, batch 64"
    if workload == "qv_plain":
        n = args.qubits if args.qubits != 32 else 24
        return f"qv_plain: {n} qubits, depth {n}, seed 1000"
    if workload == "noisy":
        from qsim_b200 import workloads as W
        from qsim_b200.circuit import NOISE_OPS, from_qiskit
        n = args.qubits if args.qubits != 32 else 12
        T = args.circuits if args.circuits != 4096 else 8192
        nn = sum(1 for ins in from_qiskit(W.noisy_brickwork(n, 8, seed=5)).data if ins.name in NOISE_OPS)
        return (f"noisy: {n}-qubit brickwork x 8 layers, {nn} channels (depolarizing, amplitude damping, "
                f"dephasing at 1e-3), {T} trajectories per step")
    if workload == "chebyshev":
        n = args.qubits if args.qubits != 32 else 22
        return (f"chebyshev: {n} qubits, ring ZZ + X field + 20 XX+YY pairs ({2 * n + 40} Pauli terms), t = 10.0, "
                f"precision 1e-06")
    if workload == "micro":
        return ("micro: 20-qubit kernels through blackwell_kernels (CUDA-tensor gates), and QV-20 (depth 20, "
                "seed 20) with 8192 shots through BlackwellSimulator.run")
    raise ValueError(workload)


# ------------------------------------------------------------ workloads
def _cuda_time(fn, stream, steps):
    import torch
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        fn()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    return ev0.elapsed_time(ev1) / 1000.0


def bench_layers32(args, dev):
    import numpy as np
    import torch
    from qsim_b200 import engine as E
    from qsim_b200 import workloads as W
    n, layers = args.qubits, 20
    ops = W.layers_ops(n, layers, seed=0)
    ngates = len(ops)
    plan = E.Plan(n, ops, dev)
    state = E.empty_state(n, f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    h = E._h(dev)
    step = lambda: plan.execute_from_zero(state)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    l0 = h.launches()
    with ClockSampler(dev) as clk:
        t = _cuda_time(step, stream, args.steps)
    launches = (h.launches() - l0)
    t = reduce_max(t, f"cuda:{dev}")
    info = plan.refresh_info()
    P = info["n_passes"]
    kernel = ("qs_tile_pass (one NVRTC-specialised kernel per pass)" if info["n_jit_passes"] == P
              else "k_pass (generic tile-pass interpreter)")
    algo_bytes = (8.0 + 16.0 * (P - 1)) * (1 << n)  # first pass writes only
    per_step = t / args.steps
    peak, src = measured_peaks()
    achieved = algo_bytes / per_step / 1e9
    # e2e: public call path with host buffers, every step
    ops_host = np.ascontiguousarray(ops)
    shots = 1024

    def e2e_step():
        p = E.Plan(n, ops_host, dev)           # host ops -> FP64 plan -> H2D program
        p.execute_from_zero(state)
        s = E.sample(state, shots).cpu()       # D2H of the result
        del p
        return s

    e2e_step()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        e2e_step()
    torch.cuda.synchronize()
    te = reduce_max((time.perf_counter() - t0) / max(1, args.steps // 2), f"cuda:{dev}")
    plan_bytes = int(plan.info["n_ops_in"]) * 304
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    res = {
        "metric": METRIC, "value": ws * ngates / per_step, "unit": "gates/s",
        "ms_per_step": per_step * 1e3, "dtype": "c64 (fp32 FMA; fp64 host fusion)",
        "config": {"workload": describe("layers32", args),
                   "passes": P, "tile_bits": info["tile_bits"], "blocks": info["n_blocks"],
                   "fused_ops": info["n_ops_fused"], "specialised_passes": info["n_jit_passes"],
                   "l2": "state 32 GiB >> 126 MB L2 (no flush needed)"},
        "hbm_gbs": achieved,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     # dram read+write per launch from the ncu capture of the
                     # same kernel at 26 qubits (537.0 + 478.6 MB), scaled by
                     # the amplitudes per launch (traffic grows in proportion)
                     "traffic": (537.0e6 + 478.6e6) * 2.0 ** (n - 26) if n >= 26 else None,
                     "traffic_source": "ncu dram__bytes_read/write.sum, 26-qubit capture scaled by 2^(n-26)",
                     "kernel": kernel, "peak_source": src,
                     "algorithmic_bytes_per_launch": algo_bytes / P},
        "e2e": {"value": ws * ngates / te, "unit": "gates/s", "h2d_bytes_per_step": plan_bytes,
                "d2h_bytes_per_step": shots * 8},
        "gpu_launches": int(launches // max(1, args.steps)) * args.steps,
        "clocks": clk.summary(),
    }
    return res, {"n": n, "ops": ops, "unit": "gates/s", "ngates": ngates}


def bench_qv_batch(args, dev):
    import ctypes as ct
    import numpy as np
    import torch
    from qsim_b200 import engine as E
    from qsim_b200 import workloads as W
    C = args.circuits
    widths, oo, ops, so = W.qv_batch(C, 10, 20, seed=1)
    t_tune = time.perf_counter()
    if args.tune_table:   # a recorded table (profiling: the tuner's own timings are distorted under a profiler)
        tuned = {int(k): tuple(v) for k, v in json.loads(args.tune_table).items()}
        E.autotune_set(tuned, dev)
    else:
        tuned = E.autotune_batch(widths, oo, ops, dev)   # shared by the batch and the per-circuit plans
    t_tune = time.perf_counter() - t_tune
    bp = E.BatchPlan(widths, oo, ops, so, dev)
    states = bp.alloc_states()
    stream = torch.cuda.current_stream(dev)
    h = E._h(dev)
    step = lambda: bp.execute(states)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    l0 = h.launches()
    with ClockSampler(dev) as clk:
        t = _cuda_time(step, stream, args.steps)
    launches = h.launches() - l0
    t = reduce_max(t, f"cuda:{dev}")
    per_step = t / args.steps
    peak, src = measured_peaks()
    achieved = bp.info["bytes_moved"] / per_step / 1e9
    # the same batch as one persistent launch (qs_set_batch_queue)
    h.call("qs_set_batch_queue", 1)
    try:
        bq = E.BatchPlan(widths, oo, ops, so, dev)
    finally:
        h.call("qs_set_batch_queue", 0)
    stepq = lambda: bq.execute(states)
    for _ in range(args.warmup):
        stepq()
    tq = reduce_max(_cuda_time(stepq, stream, args.steps), f"cuda:{dev}") / args.steps
    del bq
    # the same batch with every pass on the CUDA cores (qs_set_tensor_cores 0)
    h.call("qs_set_tensor_cores", 0)
    try:
        bc = E.BatchPlan(widths, oo, ops, so, dev)
    finally:
        h.call("qs_set_tensor_cores", 1)
    stepc = lambda: bc.execute(states)
    for _ in range(args.warmup):
        stepc()
    tcc = reduce_max(_cuda_time(stepc, stream, args.steps), f"cuda:{dev}") / args.steps
    del bc
    for _ in range(2):
        step()   # leave the states as the headline plan computes them
    # plain per-circuit path on a sample of the same circuits
    idx = np.random.default_rng(2).choice(C, size=min(64, C), replace=False)
    plans = [(int(widths[c]), E.Plan(int(widths[c]), ops[oo[c]:oo[c + 1]], dev)) for c in idx]
    bufs = [E.empty_state(w, f"cuda:{dev}") for w, _ in plans]
    for (w, p), b in zip(plans, bufs):
        p.execute_from_zero(b)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for (w, p), b in zip(plans, bufs):
        p.execute_from_zero(b)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_plain = ev0.elapsed_time(ev1) / 1000.0
    plain_cps = len(idx) / t_plain
    # the reference's plain path: one launch per gate (state init + every
    # U(4) through qs_apply_2q), on the same sample of circuits
    hdl = E._h(dev)
    mats = [[np.ascontiguousarray(np.asarray(r["m"][:32], dtype=np.float32)) for r in ops[oo[c]:oo[c + 1]]]
            for c in idx]

    def per_gate():
        for (w, _), b, c, ms in zip(plans, bufs, idx, mats):
            hdl.call("qs_state_init", ct.c_void_p(b.data_ptr()), int(w))
            for r, m in zip(ops[oo[c]:oo[c + 1]], ms):
                hdl.call("qs_apply_2q", ct.c_void_p(b.data_ptr()), int(w),
                         m.ctypes.data_as(ct.POINTER(ct.c_float)), int(r["q"][0]), int(r["q"][1]))

    per_gate()
    torch.cuda.synchronize()
    ev0.record(stream)
    per_gate()
    ev1.record(stream)
    torch.cuda.synchronize()
    pergate_cps = len(idx) / (ev0.elapsed_time(ev1) / 1000.0)
    # e2e: host ops -> one-shot batch (FP64 fusion and H2D of each slice
    # overlapping the GPU's run of the previous one) -> the state of circuit 0
    # back to the host, every step
    ops_host = np.ascontiguousarray(ops)

    def e2e_step():
        E.batch_run(widths, oo, ops_host, so, states)
        return states[: 1 << int(widths[0])].cpu()

    e2e_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ne = max(3, args.steps)   # ~0.15 s each: several steps for a stable wall-clock figure
    for _ in range(ne):
        e2e_step()
    torch.cuda.synchronize()
    te = reduce_max((time.perf_counter() - t0) / ne, f"cuda:{dev}")
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    res = {
        "metric": METRIC, "value": ws * C / per_step, "unit": "circuits/s", "ms_per_step": per_step * 1e3,
        "dtype": "c64 (fp32 FMA; fp64 host fusion)",
        "config": {"workload": describe("qv_batch", args),
                   "launches_per_step": bp.info["n_launches"], "items": bp.info["n_items"],
                   "autotuned_tile_block_bits": {str(k): list(v) for k, v in tuned.items()},
                   "autotune_seconds": t_tune, "cuda_graph": "captured at the 2nd execution, replayed",
                   "max_passes": bp.info["max_passes"], "tensor_core_launches": bp.info["n_tc_launches"],
                   "l2": "6.2 GB of states >> L2"},
        "persistent_launch": {"value": ws * C / tq, "unit": "circuits/s", "ms_per_step": tq * 1e3,
                              "note": "the same batch plan as one persistent launch (tiles taken from a device "
                                      "counter level by level); value above: one launch per pass level and tile "
                                      "shape"},
        "cuda_cores": {"value": ws * C / tcc, "unit": "circuits/s", "ms_per_step": tcc * 1e3,
                       "note": "the same batch with every pass on the CUDA-core interpreter; value above: dense "
                               "passes with 5-qubit blocks and 12/13-qubit tiles on tcgen05.mma (TF32 split)"},
        "per_circuit_launches": {"value": plain_cps, "unit": "circuits/s",
                                 "sample": f"{len(idx)} random circuits of the batch, one fused plan per circuit"},
        "per_gate_launches": {"value": pergate_cps, "unit": "circuits/s",
                              "sample": f"the same {len(idx)} circuits, one launch per gate (the reference's "
                                        f"dispatch: state init + qs_apply_2q per U(4))"},
        "hbm_gbs": achieved,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "k_pass<R> (generic tile-pass kernel, batched items)",
                     "peak_source": src},
        "e2e": {"value": ws * C / te, "unit": "circuits/s", "h2d_bytes_per_step": int(ops.nbytes),
                "d2h_bytes_per_step": 8 << int(widths[0]),
                "note": "host op records in, one-shot qs_batch_run (slices planned while the GPU runs the "
                        "previous one), state of circuit 0 out"},
        "gpu_launches": int(launches // max(1, args.steps)) * args.steps,
        "clocks": clk.summary(),
    }
    return res, {"unit": "circuits/s"}


def bench_qv12(args, dev):
    import numpy as np
    import torch
    from qsim_b200 import engine as E
    from qsim_b200 import workloads as W
    ops = W.qv_ops(12, 12, 0)
    plan = E.Plan(12, ops, dev)
    state = E.empty_state(12, f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    step = lambda: plan.execute_from_zero(state)
    for _ in range(args.warmup):
        step()
    with ClockSampler(dev) as clk:
        t = _cuda_time(step, stream, args.steps)
    t = reduce_max(t, f"cuda:{dev}")
    per_step = t / args.steps
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return {"metric": METRIC, "value": ws / per_step, "unit": "circuits/s", "ms_per_step": per_step * 1e3,
            "dtype": "c64", "config": {"workload": describe("qv12", args)},
            "clocks": clk.summary(), "gpu_launches": args.steps}, {"unit": "circuits/s"}


class ServingMix:
    """The serving request mix, seeded: 50% Quantum-Volume circuits (widths
    10-28, depth = width, 1024 shots), 25% ansatz energy+gradient requests
    (EfficientSU2, 4 reps, 12-22 qubits, 256-term observable), 25% Chebyshev
    evolutions (ring ZZ + X field + 20 random XX+YY pairs, 12-22 qubits,
    t ~ U[0.5, 10], seeded product state, precision 1e-6).  Observables,
    Hamiltonians and product states are drawn once per width."""

    def __init__(self, n_req: int, seed: int):
        import numpy as np
        self.rng = np.random.default_rng(seed)
        r = self.rng
        self.specs = []
        for i in range(n_req):
            u = r.random()
            if u < 0.5:
                self.specs.append(("qv", int(r.integers(10, 29)), 1_000_000 + i))
            elif u < 0.75:
                self.specs.append(("grad", int(r.integers(12, 23)), 2_000_000 + i))
            else:
                self.specs.append(("evo", int(r.integers(12, 23)), 3_000_000 + i, float(r.uniform(0.5, 10.0))))
        self._cache = {}

    def _per_width(self, kind, w):
        from qsim_b200 import workloads as W
        from qsim_b200.circuit import lower
        key = (kind, w)
        if key not in self._cache:
            if kind == "grad":
                qc, npar = W.efficient_su2(w, reps=4)
                self._cache[key] = (lower(qc), npar, W.random_pauli_observable(w, 256, seed=w))
            else:
                self._cache[key] = (W.serving_hamiltonian(w, seed=w), W.product_state(w, seed=w))
        return self._cache[key]

    def request(self, i):
        import numpy as np
        from qsim_b200 import workloads as W
        from qsim_b200.server import CircuitRequest, EvolutionRequest, GradientRequest
        sp = self.specs[i]
        if sp[0] == "qv":
            return CircuitRequest(n_qubits=sp[1], ops=W.qv_ops(sp[1], sp[1], sp[2]), shots=1024, seed=sp[2])
        if sp[0] == "grad":
            ops, npar, obs = self._per_width("grad", sp[1])
            p = np.random.default_rng(sp[2]).uniform(0, 2 * math.pi, (1, npar))
            return GradientRequest(n_qubits=sp[1], ops=ops, n_params=npar, params=p, observable=obs)
        ham, psi0 = self._per_width("evo", sp[1])
        return EvolutionRequest(hamiltonian=ham, t=sp[3], psi0=psi0, precision=1e-6)

    @staticmethod
    def host_bytes(req):
        import numpy as np
        b = int(np.asarray(getattr(req, "ops", np.zeros(0))).nbytes)
        if getattr(req, "psi0", None) is not None:
            b += int(np.asarray(req.psi0).size) * 8
        return b


def run_serial(mix, reqs, dev, per_gate=False):
    """The plain path, one request after the other on one stream: a plan per
    circuit + sampling, adjoint gradient, Chebyshev evolution.  per_gate: each
    circuit instead as the reference dispatches it (simulator.py:439-468 of
    the reference): state init, then one launch per gate (qs_apply_2q for
    every U(4) of the QV circuits)."""
    import ctypes as ct
    import numpy as np
    import torch
    from blackwell_backend.chebyshev import chebyshev_evolve_pauli
    from qsim_b200 import engine as E
    from qsim_b200.server import CircuitRequest, GradientRequest
    hdl = E._h(dev)
    for r in reqs:
        if isinstance(r, CircuitRequest) and per_gate:
            st = E.empty_state(r.n_qubits, f"cuda:{dev}")
            hdl.call("qs_state_init", ct.c_void_p(st.data_ptr()), int(r.n_qubits))
            for rec in r.ops:
                m = np.ascontiguousarray(np.asarray(rec["m"][:32], dtype=np.float32))
                hdl.call("qs_apply_2q", ct.c_void_p(st.data_ptr()), int(r.n_qubits),
                         m.ctypes.data_as(ct.POINTER(ct.c_float)), int(rec["q"][0]), int(rec["q"][1]))
            g = torch.Generator(device=f"cuda:{dev}")
            g.manual_seed(int(r.seed))
            E.sample(st, r.shots, generator=g).cpu()
            del st
        elif isinstance(r, CircuitRequest):
            p = E.Plan(r.n_qubits, r.ops, dev)
            st = E.empty_state(r.n_qubits, f"cuda:{dev}")
            p.execute_from_zero(st)
            g = torch.Generator(device=f"cuda:{dev}")
            g.manual_seed(int(r.seed))
            E.sample(st, r.shots, generator=g).cpu()
            del p, st
        elif isinstance(r, GradientRequest):
            E.adjoint_gradient(r.n_qubits, r.ops, r.n_params, np.asarray(r.params), r.observable, dev)
        else:
            psi = torch.as_tensor(np.asarray(r.psi0, dtype=np.complex64)).to(f"cuda:{dev}")
            out, _ = chebyshev_evolve_pauli(psi, r.hamiltonian, r.t, precision=r.precision)
            out.cpu()


def bench_serving(args, dev):
    """Poisson request streams at each rate of the sweep, served by the
    continuous-batching server (150 GB budget); the same request sequence is
    replayed at every rate.  value = served requests/s at the highest rate
    (the server saturated); p50/p99 per rate; the same requests run one by one
    on the plain path give the serial comparison."""
    import numpy as np
    import torch
    from qsim_b200 import engine as E
    from qsim_b200.server import CircuitRequest, NativeServer, Server
    make_server = NativeServer if args.server == "native" else Server
    rates = [float(x) for x in args.rates.split(",")]
    n_req = args.requests
    mix = ServingMix(n_req, seed=4)
    reqs = [mix.request(i) for i in range(n_req)]
    gaps = np.random.default_rng(5).exponential(1.0, n_req)
    unit_arrivals = np.cumsum(gaps) - gaps[0]
    h2d = sum(ServingMix.host_bytes(r) for r in reqs)
    d2h = sum((r.shots * 8 if isinstance(r, CircuitRequest) else 8 << getattr(r, "n_qubits", 0))
              for r in reqs)
    # warm-up: one request of each kind and width class through the server
    srv = make_server(device=dev, workers=args.workers)
    warm = [mix.request(i) for i in range(min(n_req, 3 * max(1, args.warmup)))]
    for f in [srv.submit(r) for r in warm]:
        f.result(600)
    srv.close()
    torch.cuda.synchronize()
    sweep = []
    stream = torch.cuda.current_stream(dev)
    L = E._h(dev).L
    with ClockSampler(dev) as clk:
        for lam in rates:
            arrivals = unit_arrivals / lam
            srv = make_server(device=dev, workers=args.workers)
            futs = [None] * n_req
            lr0 = int(L.qs_launch_count(None))
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            barrier()
            ev0.record(stream)
            t0 = time.perf_counter()
            for i, r in enumerate(reqs):
                dt = arrivals[i] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                futs[i] = srv.submit(r)
            for f in futs:
                f.result(1800)
            torch.cuda.synchronize()
            ev1.record(stream)
            torch.cuda.synchronize()
            makespan = ev0.elapsed_time(ev1) / 1000.0
            st = srv.stats()
            srv.close()
            kinds = np.array([sp[0] for sp in mix.specs])
            qv_n = int((kinds == "qv").sum())
            sweep.append({"rate_rps": lam, "served_rps": n_req / makespan, "qv_circuits_per_s": qv_n / makespan,
                          "p50_ms": float(st["p50_ms"]), "p99_ms": float(st["p99_ms"]),
                          "makespan_s": makespan, "offered_s": float(arrivals[-1]),
                          "gpu_launches": int(L.qs_launch_count(None)) - lr0})
    # serial plain execution of the same requests
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    run_serial(mix, reqs, dev)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_serial = ev0.elapsed_time(ev1) / 1000.0
    # the same, with each circuit dispatched one launch per gate (the
    # reference's per-circuit launch sequence)
    torch.cuda.synchronize()
    ev0.record(stream)
    run_serial(mix, reqs, dev, per_gate=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_serial_pg = ev0.elapsed_time(ev1) / 1000.0
    top = sweep[-1]
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    top_mk = reduce_max(top["makespan_s"], f"cuda:{dev}")
    res = {
        "metric": METRIC, "value": ws * n_req / top_mk, "unit": "requests/s",
        "ms_per_step": top_mk * 1e3, "dtype": "c64 state (fp32 FMA), fp64 reductions",
        "config": {"workload": describe("serving", args),
                   "rates_rps": rates, "step": "one replay of the request sequence at the highest rate",
                   "l2": "states up to 2 GiB each; no flush"},
        "sweep": sweep,
        "served_circuits_per_s": ws * top["qv_circuits_per_s"],
        "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"],
        "serial_plain": {"value": n_req / t_serial, "unit": "requests/s", "seconds": t_serial,
                         "speedup": t_serial / top["makespan_s"],
                         "note": "one request after the other, each circuit as one fused plan"},
        "serial_per_gate": {"value": n_req / t_serial_pg, "unit": "requests/s", "seconds": t_serial_pg,
                            "speedup": t_serial_pg / top["makespan_s"],
                            "note": "one request after the other, each circuit as the reference dispatches it: "
                                    "one launch per gate"},
        "e2e": {"value": ws * n_req / top_mk, "unit": "requests/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h),
                "note": "host request -> admission -> device -> host result; the value itself is end to end"},
        "gpu_launches": top["gpu_launches"],
        "clocks": clk.summary(),
    }
    return res, {"unit": "requests/s"}


def bench_adjoint(args, dev):
    """Energy and full gradient of a 20-qubit EfficientSU2 ansatz (4 reps,
    200 parameters) for a batch of 64 parameter vectors, observable = 256
    random Pauli strings of weight 1-4.  value = gradient evaluations
    (parameter vectors) per second through the adjoint kernels; the forward
    (energies only: batched circuits + <H>) is timed on the same batch for the
    backward/forward ratio."""
    import numpy as np
    import torch
    from qsim_b200 import engine as E
    from qsim_b200 import workloads as W
    from qsim_b200.circuit import lower
    n, B = args.qubits if args.qubits != 32 else 20, 64
    qc, npar = W.efficient_su2(n, reps=4)
    ops = lower(qc)
    obs = W.random_pauli_observable(n, 256, seed=3)
    params = np.random.default_rng(8).uniform(0, 2 * math.pi, (B, npar))
    stream = torch.cuda.current_stream(dev)
    pidx = ops["param"].astype(np.int64)

    def forward():
        bound = np.concatenate([ops] * B)
        for b in range(B):
            blk = bound[b * len(ops):(b + 1) * len(ops)]
            sel = pidx >= 0
            blk["m"][sel, 0] = params[b, pidx[sel]]
        widths = np.full(B, n, dtype=np.int32)
        oo = np.arange(B + 1, dtype=np.int64) * len(ops)
        so = np.arange(B, dtype=np.int64) << n
        bp = E.BatchPlan(widths, oo, bound, so, dev)
        st = bp.alloc_states()
        bp.execute(st)
        return [E.expect_pauli_sum(st[b << n:(b + 1) << n], obs) for b in range(B)]

    def gradient():
        return E.adjoint_gradient(n, ops, npar, params, obs, dev)

    for _ in range(args.warmup):
        forward()
        gradient()
    h = E._h(dev)
    with ClockSampler(dev) as clk:
        t_f = _cuda_time(forward, stream, args.steps) / args.steps
        l0 = h.launches()
        t_g = _cuda_time(gradient, stream, args.steps) / args.steps
        launches = h.launches() - l0
    t_f, t_g = reduce_max(t_f, f"cuda:{dev}"), reduce_max(t_g, f"cuda:{dev}")
    e_f = np.array(forward())
    e_g, g = gradient()
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    amp = B << n
    return {"metric": METRIC, "value": ws * B / t_g, "unit": "gradients/s", "ms_per_step": t_g * 1e3,
            "dtype": "c64 state, fp64 gradient accumulation",
            "config": {"workload": describe("adjoint", args), "l2": f"{amp * 8 >> 20} MiB of states per batch > L2"},
            "forward_ms": t_f * 1e3, "gradient_over_forward": t_g / t_f,
            "energy_agreement": float(np.max(np.abs(e_f - e_g))),
            "e2e": {"value": ws * B / t_g, "unit": "gradients/s", "h2d_bytes_per_step": int(params.nbytes + ops.nbytes),
                    "d2h_bytes_per_step": int(g.nbytes + e_g.nbytes),
                    "note": "host parameters in, host FP64 gradients out, every step"},
            "gpu_launches": int(launches // max(1, args.steps)) * args.steps, "clocks": clk.summary()}, \
        {"unit": "gradients/s"}


def bench_qv_plain(args, dev):
    """One Quantum-Volume circuit of --qubits qubits (depth = width, seed
    1000) on the plain per-circuit path: one plan, executed from |0> each
    step (specialisation as --jit says).  value = circuits/s."""
    import torch
    from qsim_b200 import engine as E
    from qsim_b200 import workloads as W
    n = args.qubits if args.qubits != 32 else 24
    ops = W.qv_ops(n, n, 1000)
    plan = E.Plan(n, ops, dev)
    state = E.empty_state(n, f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    h = E._h(dev)
    step = lambda: plan.execute_from_zero(state)
    for _ in range(args.warmup):
        step()
    l0 = h.launches()
    with ClockSampler(dev) as clk:
        t = _cuda_time(step, stream, args.steps)
    launches = h.launches() - l0
    t = reduce_max(t, f"cuda:{dev}")
    per_step = t / args.steps
    info = plan.refresh_info()
    peak, src = measured_peaks()
    algo = (8.0 + 16.0 * (info["n_passes"] - 1)) * (1 << n)
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return {"metric": METRIC, "value": ws / per_step, "unit": "circuits/s", "ms_per_step": per_step * 1e3,
            "dtype": "c64", "config": {"workload": describe("qv_plain", args),
                                       "passes": info["n_passes"], "specialised_passes": info["n_jit_passes"]},
            "roofline": {"bound": "hbm", "achieved": algo / per_step / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": algo / per_step / 1e9 / peak, "traffic": None, "peak_source": src},
            "clocks": clk.summary(), "gpu_launches": launches}, {"unit": "circuits/s"}


def _per_channel_trajectories(qc, n_traj, dev):
    """Trajectories/s through the reference's one-call-per-gate-or-channel
    API (blackwell_kernels: apply_gate / apply_mcgate per gate, one
    apply_depolarizing / apply_amplitude_damping / apply_dephasing call per
    channel, each state-dependent one returning its branch to the host, as
    the reference's do).  Gate matrices are built before timing."""
    import time as _t
    import numpy as np
    import torch
    import blackwell_kernels as bk
    from qsim_b200 import gates as G
    calls = []
    xg = torch.tensor([[0, 1], [1, 0]], dtype=torch.complex64, device=f"cuda:{dev}")
    for ins in qc.data:
        if ins.name in ("ry", "rz"):
            m = torch.tensor(G.mat1(ins.name, ins.params), dtype=torch.complex64, device=f"cuda:{dev}")
            calls.append((bk.apply_gate, m, ins.qubits[0]))
        elif ins.name == "cx":
            calls.append((bk.apply_mcgate, xg, [ins.qubits[0]], ins.qubits[1]))
        elif ins.name == "depolarize":
            calls.append((bk.apply_depolarizing, ins.qubits[0], ins.params[0]))
        elif ins.name == "amplitude_damp":
            calls.append((bk.apply_amplitude_damping, ins.qubits[0], ins.params[0]))
        elif ins.name == "dephase":
            calls.append((bk.apply_dephasing, ins.qubits[0], ins.params[0]))
    torch.cuda.synchronize()
    t0 = _t.perf_counter()
    for _ in range(n_traj):
        st = bk.state_init(qc.num_qubits)
        for c in calls:
            c[0](st, *c[1:])
    torch.cuda.synchronize()
    return n_traj / (_t.perf_counter() - t0)


def bench_noisy(args, dev):
    """Noise trajectories: a --qubits (default 12) qubit brickwork of 8 layers
    (RY, RZ on every qubit, CX pairs) with depolarizing, amplitude-damping
    and dephasing channels (1e-3 each) after every gate on each of its
    qubits; --circuits trajectories (default 8192) per step, seeds advancing
    every step.  value = trajectories/s of qs_noise_trajectories with the
    seeds and circuit on the host and the states left on the device; e2e
    also copies every channel's branch back to the host.  Compared with the
    reference-style path: one API call per gate and per channel."""
    import numpy as np
    import torch
    from qsim_b200 import engine as E
    from qsim_b200 import workloads as W
    from qsim_b200.noise import n_channels, run_trajectories
    n = args.qubits if args.qubits != 32 else 12
    T = args.circuits if args.circuits != 4096 else 8192
    qc = W.noisy_brickwork(n, 8, seed=5)
    nn = n_channels(qc)
    out = torch.empty((T, 1 << n), dtype=torch.complex64, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    h = E._h(dev)
    k = [0]

    def step(branches=False):
        k[0] += 1
        return run_trajectories(qc, T, seed=k[0] * T, out=out, branches=branches)

    for _ in range(args.warmup):
        step()
    l0 = h.launches()
    with ClockSampler(dev) as clk:
        t = _cuda_time(step, stream, args.steps)
        launches = h.launches() - l0
        t_e2e = _cuda_time(lambda: step(True), stream, args.steps)
    t, t_e2e = reduce_max(t, f"cuda:{dev}"), reduce_max(t_e2e, f"cuda:{dev}")
    per_step, per_e2e = t / args.steps, t_e2e / args.steps
    ref_rate = _per_channel_trajectories(qc, 2, dev)
    peak, src = measured_peaks()
    algo = 8.0 * T * (1 << n)   # one level: each trajectory's state written once
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return {"metric": METRIC, "value": ws * T / per_step, "unit": "trajectories/s", "ms_per_step": per_step * 1e3,
            "dtype": "c64 state, fp64 branch probabilities",
            "config": {"workload": describe("noisy", args),
                       "l2": f"{(T << n) * 8 >> 20} MiB of states per step"},
            "per_channel_launches": {"value": ref_rate, "unit": "trajectories/s",
                                     "note": "one blackwell_kernels call per gate and per channel"},
            "roofline": {"bound": "hbm", "achieved": algo / per_step / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": algo / per_step / 1e9 / peak, "traffic": None, "peak_source": src,
                         "note": "the whole circuit runs in shared memory; HBM only sees each final state once, "
                                 "so this fraction is low by design (the work is shared-memory sweeps)"},
            "e2e": {"value": ws * T / per_e2e, "unit": "trajectories/s", "h2d_bytes_per_step": int(T * 64),
                    "d2h_bytes_per_step": int(T * nn),
                    "note": "item table (state offset, seed, branch slot per trajectory) in, every branch out; "
                            "the shared program (a few hundred KB) is uploaded too"},
            "clocks": clk.summary(), "gpu_launches": int(launches)}, {"unit": "trajectories/s"}


def bench_chebyshev(args, dev):
    """Chebyshev evolution exp(-iHt)|psi> at the largest size of the serving
    mix's evolution requests: --qubits (default 22) qubits, H = ring J ZZ +
    h X field + 20 random K (XX + YY) pairs (seed n), t = 10, precision 1e-6,
    seeded product state.  value = evolutions/s of the matrix-free path
    (chebyshev_evolve_pauli) on a resident state; e2e = host state in, host
    state out.  The CSR path with the reference's algorithm (chebyshev_evolve
    over a CSR of the same H) is timed beside it.  Roofline per degree:
    matrix-free 40 N bytes (read x_k, x_(k-1) and the accumulator, write
    x_(k+1) and the accumulator); CSR 12 nnz + 4 (N+1) + 40 N."""
    import numpy as np
    import torch
    from blackwell_backend.chebyshev import chebyshev_evolve, chebyshev_evolve_pauli
    from blackwell_backend.hamiltonian import HamiltonianCSR
    from qsim_b200 import workloads as W
    from qsim_b200.paulis import csr_from_paulis
    n = args.qubits if args.qubits != 32 else 22
    N = 1 << n
    t_evo, prec = 10.0, 1e-6
    H = W.serving_hamiltonian(n, seed=n)
    psi_h = np.ascontiguousarray(W.product_state(n, seed=n).astype(np.complex64))
    psi = torch.from_numpy(psi_h).to(f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    res_pf = {}

    def step_pf():
        res_pf["out"], res_pf["info"] = chebyshev_evolve_pauli(psi, H, t_evo, precision=prec)

    for _ in range(args.warmup):
        step_pf()
    from qsim_b200 import engine as E
    h = E._h(dev)
    l0 = h.launches()
    with ClockSampler(dev) as clk:
        t_pf = _cuda_time(step_pf, stream, args.steps)
        launches = h.launches() - l0

        def step_e2e():
            d = torch.from_numpy(psi_h).to(f"cuda:{dev}", non_blocking=False)
            o, _ = chebyshev_evolve_pauli(d, H, t_evo, precision=prec)
            return o.cpu()

        t0 = time.perf_counter()
        for _ in range(args.steps):
            step_e2e()
        torch.cuda.synchronize()
        t_e2e = time.perf_counter() - t0
    K = int(res_pf["info"]["chebyshev_degree"])
    # the CSR path (reference algorithm) on the same H
    row_ptr, col, val = csr_from_paulis(H)
    nnz = int(row_ptr[-1])
    csr = HamiltonianCSR(torch.from_numpy(row_ptr).to(f"cuda:{dev}"), torch.from_numpy(col).to(f"cuda:{dev}"),
                         torch.from_numpy(val).to(f"cuda:{dev}"), n, H.spectral_bound(), paulis=H)
    res_csr = {}

    def step_csr():
        res_csr["out"], res_csr["info"] = chebyshev_evolve(psi, csr, t_evo, precision=prec)

    step_csr()
    t_csr = _cuda_time(step_csr, stream, max(1, args.steps))
    a = res_pf["out"].cpu().numpy().astype(np.complex128)
    b = res_csr["out"].cpu().numpy().astype(np.complex128)
    fid = float(abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real))
    t_pf, t_csr, t_e2e = (reduce_max(x, f"cuda:{dev}") for x in (t_pf, t_csr, t_e2e))
    per, per_csr, per_e2e = t_pf / args.steps, t_csr / max(1, args.steps), t_e2e / args.steps
    peak, src = measured_peaks()
    algo_pf = 40.0 * N                                   # bytes per degree
    algo_csr = 12.0 * nnz + 4.0 * (N + 1) + 40.0 * N
    ach_pf = algo_pf * K / per / 1e9
    ach_csr = algo_csr * K / per_csr / 1e9
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return {"metric": METRIC, "value": ws / per, "unit": "evolutions/s", "ms_per_step": per * 1e3,
            "dtype": "c64 vectors (fp32 FMA), fp64 Bessel coefficients",
            "config": {"workload": describe("chebyshev", args), "degree": K,
                       "l2": f"3 vectors of {(8 * N) >> 20} MiB (the recurrence re-reads them every degree)"},
            "roofline": {"bound": "hbm", "achieved": ach_pf, "peak": peak, "unit": "GB/s", "frac": ach_pf / peak,
                         "traffic": None, "peak_source": src, "kernel": "k_chebp_fused (matrix-free, one per degree)",
                         "algorithmic_bytes_per_launch": algo_pf,
                         "note": "each amplitude also gathers x_k[i ^ x_t] for every Pauli term (from L2 when the "
                                 "vector fits there), so the kernel is bound by those gathers, not by its 40 N bytes"},
            "csr_path": {"value": 1.0 / per_csr, "unit": "evolutions/s", "nnz": nnz,
                         "roofline": {"achieved": ach_csr, "frac": ach_csr / peak, "unit": "GB/s",
                                      "kernel": "k_cheb_fused (CSR SpMV + step + accumulate)",
                                      "algorithmic_bytes_per_launch": algo_csr},
                         "fidelity_vs_matrix_free": fid},
            "e2e": {"value": ws / per_e2e, "unit": "evolutions/s", "h2d_bytes_per_step": 8 * N,
                    "d2h_bytes_per_step": 8 * N, "note": "host product state in, evolved state out"},
            "clocks": clk.summary(), "gpu_launches": int(launches)}, {"unit": "evolutions/s"}


# The reference's published single-kernel times at 20 qubits and its QV-20
# end-to-end time (RTX 5090; README.md:152,160-167 of the reference).
REF_MICRO_US = {"apply_gate": 4.2, "apply_gate_2q": 6.2, "apply_diagonal": 4.1, "apply_diagonal_phase": 2.1,
                "apply_mcgate": 5.0, "measure_qubit": 24.7, "sample_1000": 20.5, "apply_gates_fused_10": 10.3}
REF_QV20_E2E_MS = 126.0


def bench_micro(args, dev):
    """The operations the reference publishes times for, at 20 qubits (an
    8 MiB state, L2-resident as in the reference's table), through the
    blackwell_kernels API with the gates as CUDA tensors: device time per
    call (CUDA events over --circuits calls, default 200, after warm-up).
    value = QV-20 (depth 20, seed 20) end to end with 8192 shots through
    BlackwellSimulator.run (plan cached after the first call), circuits/s."""
    import numpy as np
    import torch
    import blackwell_kernels as bk
    from blackwell_backend import BlackwellSimulator
    from qsim_b200 import workloads as W
    from qsim_b200.circuit import Circuit
    n = 20
    reps = args.circuits if args.circuits != 4096 else 200
    state = bk.state_init(n)
    bk.apply_gate(state, bk.hadamard_gate(), 0)
    stream = torch.cuda.current_stream(dev)
    H, U2, D = bk.hadamard_gate(), bk.random_unitary_4x4(), bk.rz_gate_diag(0.3)
    X = bk.pauli_x_gate()
    gates10 = torch.stack([bk.random_unitary() for _ in range(10)])
    targets10 = torch.arange(10, dtype=torch.int32, device=f"cuda:{dev}") * 2
    ops = {
        "apply_gate": lambda k: bk.apply_gate(state, H, 7 + (k & 1)),
        "apply_gate_2q": lambda k: bk.apply_gate_2q(state, U2, 3, 11),
        "apply_diagonal": lambda k: bk.apply_diagonal(state, D, 9),
        "apply_diagonal_phase": lambda k: bk.apply_diagonal_phase(state, complex(0.6, 0.8), 9),
        "apply_mcgate": lambda k: bk.apply_mcgate(state, X, [2, 5], 14),
        "measure_qubit": lambda k: bk.measure_qubit(bk.apply_gate(state, H, 4), 4, 0.5),
        "sample_1000": lambda k: bk.sample(state, 1000),
        "apply_gates_fused_10": lambda k: bk.apply_gates_fused(state, gates10, targets10),
    }
    out = {}
    for name, fn in ops.items():
        for k in range(5):
            fn(k)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        for k in range(reps):
            fn(k)
        ev1.record(stream)
        torch.cuda.synchronize()
        us = ev0.elapsed_time(ev1) * 1e3 / reps
        if name == "measure_qubit":
            us -= out["apply_gate"]["b200_us"]  # each call re-mixes qubit 4 with one H first
        out[name] = {"b200_us": us, "reference_rtx5090_us": REF_MICRO_US[name]}
    # sampling from a state far past L2: 1024 shots from 30 qubits (8 GiB).
    # One call reads the state once (chunk sums), scans the 2^19 chunk sums
    # and searches one chunk per shot; its floor is the 8 N-byte read.
    nw, shots_w = 30, 1024
    wide = bk.state_init(nw)
    for q in range(0, nw, 3):
        bk.apply_gate(wide, H, q)
    for _ in range(3):
        bk.sample(wide, shots_w)
    reps_w = 10
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(reps_w):
        bk.sample(wide, shots_w)
    ev1.record(stream)
    torch.cuda.synchronize()
    us = ev0.elapsed_time(ev1) * 1e3 / reps_w
    peak, peak_kind = measured_peaks()
    floor_us = (8 << nw) / (peak * 1e9) * 1e6
    out["sample_1024_at_30_qubits"] = {"b200_us": us, "hbm_floor_us": floor_us, "frac": floor_us / us,
                                       "peak": f"{peak} GB/s copy ({peak_kind})"}
    del wide
    torch.cuda.empty_cache()
    # QV-20 end to end
    qv = W.qv_ops(n, n, 20)
    qc = Circuit(n, n, name="qv20")
    for r in qv:
        m = (np.asarray(r["m"][:32]).reshape(16, 2) @ np.array([1, 1j])).reshape(4, 4)
        qc.unitary(m, [int(r["q"][0]), int(r["q"][1])])
    for q in range(n):
        qc.measure(q, q)
    sim = BlackwellSimulator(device=f"cuda:{dev}")
    for _ in range(max(1, args.warmup)):
        sim.run(qc, shots=8192, seed=1)
    times = []
    l0 = E_launches(dev)
    with ClockSampler(dev) as clk:
        for k in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = sim.run(qc, shots=8192, seed=k)
            _ = res.get_counts()
            times.append(time.perf_counter() - t0)
    launches = E_launches(dev) - l0
    t = reduce_max(float(np.median(times)), f"cuda:{dev}")
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return {"metric": METRIC, "value": ws / t, "unit": "circuits/s", "ms_per_step": t * 1e3,
            "dtype": "c64 (fp32; compensated 1Q/2Q kernels), fp64 reductions",
            "config": {"workload": describe("micro", args),
                       "l2": "8 MiB state, L2-resident (as the reference's table)"},
            "kernels": out,
            "qv20_e2e": {"b200_ms": t * 1e3, "reference_rtx5090_ms": REF_QV20_E2E_MS},
            "e2e": {"value": ws / t, "unit": "circuits/s", "h2d_bytes_per_step": int(qv.nbytes),
                    "d2h_bytes_per_step": 8192 * 8,
                    "note": "host circuit in, counts out (histogram on the device)"},
            "clocks": clk.summary(), "gpu_launches": int(launches)}, {"unit": "circuits/s"}


def E_launches(dev):
    from qsim_b200 import engine as E
    return int(E._h(dev).L.qs_launch_count(None))


WORKLOADS = {"layers32": bench_layers32, "qv_batch": bench_qv_batch, "qv12": bench_qv12, "serving": bench_serving,
             "adjoint": bench_adjoint, "qv_plain": bench_qv_plain, "noisy": bench_noisy, "micro": bench_micro,
             "chebyshev": bench_chebyshev}


def headline_sub_records(args, dev) -> dict:
    """The metric's served/batched halves beside the default 32-qubit line,
    each with its own timed region and clock record: `batched` = the
    qv_batch workload (4096 QV circuits of widths 10-20 against one plan and
    one launch sequence per circuit), `serving` = the serving workload on a
    trimmed request count at three rates (p50/p99 per rate, against serial
    plain execution of the same requests)."""
    import copy
    from qsim_b200 import engine as E
    E.set_jit(1, 24, dev)   # the library default: the 32-qubit line compiled every pass first
    a = copy.copy(args)
    a.circuits, a.steps, a.warmup = 4096, max(3, min(args.steps, 5)), 3
    qb, _ = bench_qv_batch(a, dev)
    batched = {
        "workload": describe("qv_batch", a), "value": qb["value"], "unit": qb["unit"], "steps": a.steps,
        "ms_per_step": qb["ms_per_step"],
        "persistent_launch": qb["persistent_launch"],
        "per_circuit_launches": qb["per_circuit_launches"], "per_gate_launches": qb["per_gate_launches"],
        "over_per_circuit_launches": qb["value"] / qb["per_circuit_launches"]["value"],
        "over_per_gate_launches": qb["value"] / qb["per_gate_launches"]["value"],
        "e2e": qb["e2e"], "roofline": qb["roofline"], "gpu_launches": qb["gpu_launches"], "clocks": qb["clocks"],
        "launches_per_step": qb["config"].get("launches_per_step"),
    }
    a = copy.copy(args)
    a.requests, a.rates, a.workers, a.server, a.warmup = 120, "100,500,2000", 4, "native", 1
    sv, _ = bench_serving(a, dev)
    serving = {
        "workload": describe("serving", a), "value": sv["value"], "unit": sv["unit"],
        "served_circuits_per_s": sv["served_circuits_per_s"],
        "p50_ms": sv["p50_ms"], "p99_ms": sv["p99_ms"],
        "sweep": [{k: r[k] for k in ("rate_rps", "served_rps", "qv_circuits_per_s", "p50_ms", "p99_ms", "makespan_s")}
                  for r in sv["sweep"]],
        "serial_plain": sv["serial_plain"], "serial_per_gate": sv["serial_per_gate"], "e2e": sv["e2e"], "gpu_launches": sv["gpu_launches"],
        "clocks": sv["clocks"],
    }
    return {"batched": batched, "serving": serving}


# --------------------------------------------------------- CPU baseline
def _cpu_worker(kind: str, n: int, seconds: float, seed0: int):
    """One process of a parallel CPU sample (started with the spawn method):
    runs work items of `kind` for about `seconds` on one thread; returns
    (items done, elapsed seconds)."""
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"
    sys.path[:0] = [os.path.join(ROOT, "qiskit-blackwell_b200", "python"), os.path.join(ROOT, "oracle")]
    import numpy as np
    import sv_oracle as O
    from qsim_b200 import workloads as W
    if kind == "noisy":
        from qsim_b200.circuit import lower
        ops = np.ascontiguousarray(lower(W.noisy_brickwork(n, 8, seed=5)))
        t0 = time.perf_counter()
        k = 0
        while time.perf_counter() - t0 < seconds or k == 0:
            O.noise_trajectory(n, ops, seed0 + k)
            k += 1
        return k, time.perf_counter() - t0
    if kind == "chebyshev":
        import scipy.sparse as sp
        from scipy.sparse.linalg import expm_multiply
        from qsim_b200.paulis import csr_from_paulis
        H = W.serving_hamiltonian(n, seed=n)
        rp, ci, va = csr_from_paulis(H)
        A = sp.csr_matrix((va.astype(np.complex128), ci, rp), shape=(1 << n, 1 << n))
        psi = W.product_state(n, seed=n)
        t0 = time.perf_counter()
        expm_multiply(-1j * 10.0 * A, psi)
        return 1, time.perf_counter() - t0
    raise ValueError(kind)


def _parallel_rate(kind: str, n: int, seconds: float, procs: int):
    """Items per second of `procs` concurrent _cpu_worker processes:
    (total items, slowest worker's elapsed seconds)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")   # safe after CUDA initialisation
    with ctx.Pool(procs) as pool:
        res = pool.starmap(_cpu_worker, [(kind, n, seconds, 1_000_003 * w) for w in range(procs)])
    return sum(r[0] for r in res), max(r[1] for r in res)


def cpu_baseline(workload: str, args) -> dict:
    """FP64 CPU restatement (oracle/sv64.c, OpenMP, all host cores) on a
    bounded sample, scaled to the workload's unit."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import sv_oracle as O
    from qsim_b200 import workloads as W
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    if workload == "layers32":
        # the same generator at 26 qubits (1 GiB FP64 state), gates in
        # circuit order for about 8 s (at least 96 gates)
        n_s = 26
        ops = np.ascontiguousarray(W.layers_ops(n_s, 20, seed=0))
        psi = np.empty(1 << n_s, dtype=np.complex128)
        O.lib().sv64_init(psi.ctypes.data, n_s)
        done = 0
        t0 = time.perf_counter()
        while done < len(ops) and (done < 96 or time.perf_counter() - t0 < 8.0):
            chunk = np.ascontiguousarray(ops[done: done + 32])
            O.lib().sv64_apply_ops(psi.ctypes.data, n_s, chunk.ctypes.data, len(chunk))
            done += len(chunk)
        dt = time.perf_counter() - t0
        per_gate_32 = dt / done * 2 ** (args.qubits - n_s)
        return {"value": 1.0 / per_gate_32, "unit": "gates/s", "cores": cores, "kind": "port",
                "sample": f"first {done} gates of the same generator at {n_s} qubits (FP64), "
                          f"time x 2^{args.qubits - n_s} (extrapolated to {args.qubits} qubits)"}
    if workload == "micro":
        t0 = time.perf_counter()
        tot = 0
        while time.perf_counter() - t0 < 10 or tot == 0:
            psi = O.simulate(20, W.qv_ops(20, 20, 20))
            O.sample_indices(psi, np.random.default_rng(tot).random(8192))
            tot += 1
        dt = time.perf_counter() - t0
        return {"value": tot / dt, "unit": "circuits/s", "cores": cores, "kind": "port",
                "sample": f"{tot} runs of QV-20 + 8192 shots (FP64 C restatement, OpenMP)"}
    if workload == "noisy":
        n = args.qubits if args.qubits != 32 else 12
        tot, dt = _parallel_rate("noisy", n, 10.0, cores)
        return {"value": tot / dt, "unit": "trajectories/s", "cores": cores, "kind": "port",
                "sample": f"{tot} trajectories of the same circuit (FP64 numpy restatement), one process per "
                          f"core for ~10 s"}
    if workload == "serving":
        # The same request sequence executed one by one on the CPU, as a
        # model: each kind is timed at a small width and scaled per request
        # by 2^(w - w_s) and by its gate count or Chebyshev degree.
        import scipy.sparse as sp
        from scipy.sparse.linalg import expm_multiply
        from blackwell_backend.chebyshev import chebyshev_coefficients
        from qsim_b200.circuit import lower
        from qsim_b200.paulis import csr_from_paulis
        ws_ = 14
        t0 = time.perf_counter()
        psi = O.simulate(ws_, W.qv_ops(ws_, ws_, 1))
        O.sample_indices(psi, np.random.default_rng(0).random(1024))
        t_qv = time.perf_counter() - t0
        qc, npar_s = W.efficient_su2(ws_, reps=4)
        obs = W.random_pauli_observable(ws_, 256, seed=ws_)
        th = np.random.default_rng(1).uniform(0, 2 * math.pi, npar_s)
        t0 = time.perf_counter()
        O.energy(ws_, lower(qc), th, obs.x, obs.z, obs.real_coefs())
        t_en = time.perf_counter() - t0
        Hs = W.serving_hamiltonian(ws_, seed=ws_)
        rp, ci, va = csr_from_paulis(Hs)
        A = sp.csr_matrix((va.astype(np.complex128), ci, rp), shape=(1 << ws_, 1 << ws_))
        t0 = time.perf_counter()
        expm_multiply(-1j * 10.0 * A, W.product_state(ws_, seed=ws_))
        t_ev = time.perf_counter() - t0
        k_s = chebyshev_coefficients(10.0, Hs.spectral_bound(), 1e-6)[1]
        mix = ServingMix(args.requests, seed=4)
        total = 0.0
        for spc in mix.specs:
            w = spc[1]
            if spc[0] == "qv":
                total += t_qv * 2.0 ** (w - ws_) * (w / ws_) ** 2
            elif spc[0] == "grad":
                total += 2 * (10 * w) * t_en * 2.0 ** (w - ws_) * (w / ws_)
            else:
                k_w = chebyshev_coefficients(spc[3], W.serving_hamiltonian(w, seed=w).spectral_bound(), 1e-6)[1]
                total += t_ev * 2.0 ** (w - ws_) * k_w / k_s
        return {"value": len(mix.specs) / total, "unit": "requests/s", "cores": cores, "kind": "port",
                "sample": f"model of the {len(mix.specs)}-request mix run serially on the FP64 CPU restatements: "
                          f"QV + 1024 shots, one energy and one expm_multiply (t = 10) timed at {ws_} qubits, "
                          f"scaled per request by 2^(w-{ws_}) and gate count (gradients: parameter shift, 2 x "
                          f"n_params energies) or Chebyshev degree"}
    if workload == "adjoint":
        # Parameter shift on the FP64 restatement: 2 x n_params energies per
        # gradient (the reference has no gradient path; a statevector
        # simulator without adjoint support differentiates this way).
        from qsim_b200.circuit import lower
        n = args.qubits if args.qubits != 32 else 20
        qc, npar = W.efficient_su2(n, reps=4)
        ops = lower(qc)
        obs = W.random_pauli_observable(n, 256, seed=3)
        theta = np.random.default_rng(8).uniform(0, 2 * math.pi, npar)
        t0 = time.perf_counter()
        k = 0
        while time.perf_counter() - t0 < 10 or k == 0:
            O.energy(n, ops, theta, obs.x, obs.z, obs.real_coefs())
            k += 1
        per_energy = (time.perf_counter() - t0) / k
        return {"value": 1.0 / (2 * npar * per_energy), "unit": "gradients/s", "cores": cores, "kind": "port",
                "sample": f"{k} FP64 energy evaluations at {n} qubits (C restatement, OpenMP, with the numpy "
                          f"Pauli expectation), x {2 * npar} per parameter-shift gradient"}
    if workload == "chebyshev":
        # scipy's expm_multiply (the reference's FP64 Chebyshev oracle family)
        # on the same generator at 16 qubits, scaled by 2^(n-16) and by the
        # ratio of the Chebyshev degrees (work per step ~ N x degree)
        from blackwell_backend.chebyshev import chebyshev_coefficients
        n = args.qubits if args.qubits != 32 else 22
        n_s = min(n, 16)
        tot, dt = _parallel_rate("chebyshev", n_s, 0.0, cores)
        k_s = chebyshev_coefficients(10.0, W.serving_hamiltonian(n_s, seed=n_s).spectral_bound(), 1e-6)[1]
        k_n = chebyshev_coefficients(10.0, W.serving_hamiltonian(n, seed=n).spectral_bound(), 1e-6)[1]
        per = dt / tot * 2 ** (n - n_s) * k_n / k_s
        return {"value": 1.0 / per, "unit": "evolutions/s", "cores": cores, "kind": "port",
                "sample": f"scipy expm_multiply (FP64), {tot} concurrent evolutions at {n_s} qubits (one process "
                          f"per core), t = 10, x 2^{n - n_s} x degree ratio {k_n}/{k_s} (extrapolated to {n} qubits)"}
    # circuits/s workloads: QV circuits at widths drawn as in the batch
    rng = np.random.default_rng(7)
    ws_ = rng.integers(10, 21, size=24)
    t0 = time.perf_counter()
    tot = 0.0
    for i, w in enumerate(ws_):
        if workload == "qv12":
            w = 12
        O.simulate(int(w), W.qv_ops(int(w), int(w), i))
        tot += 1
        if time.perf_counter() - t0 > 20:
            break
    dt = time.perf_counter() - t0
    return {"value": tot / dt, "unit": "circuits/s", "cores": cores, "kind": "port",
            "sample": f"{int(tot)} QV circuits (FP64 C restatement, OpenMP)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="layers32", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--qubits", type=int, default=32)
    ap.add_argument("--circuits", type=int, default=4096)
    ap.add_argument("--requests", type=int, default=200, help="serving: requests per rate")
    ap.add_argument("--rates", default="50,100,200,500,1000,2000", help="serving: Poisson rates (req/s)")
    ap.add_argument("--workers", type=int, default=4, help="serving: worker streams")
    ap.add_argument("--server", default="native", choices=["native", "python"],
                    help="serving: the C++ runtime (qs_server_*) or the Python one")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sub", action="store_true",
                    help="layers32: skip the batched and serving sub-records of the headline metric")
    ap.add_argument("--tile-bits", type=int, default=0, help="planner tile bits (10..14; 0 = library default)")
    ap.add_argument("--block-bits", type=int, default=0, help="register-block qubits (2..5; 0 = default)")
    ap.add_argument("--tune-table", default="",
                    help='qv_batch: JSON {width: [tile_bits, block_bits]} recorded instead of autotuning')
    ap.add_argument("--jit", type=int, default=-1,
                    help="pass specialisation: 0 off, 1 tiered (background compile, plans >= 24 qubits), "
                         "2 before first execution (-1 = 2 for layers32, else the library default)")
    args = ap.parse_args()
    ws, rank, local = dist_env()

    if args.impl == "reference":
        if rank != 0:
            return 0
        vals = []
        info = None
        for _ in range(args.warmup):
            pass
        for _ in range(max(1, args.steps)):
            info = cpu_baseline(args.workload, args)
            vals.append(info["value"])
        v = float(sorted(vals)[len(vals) // 2])
        line = {"metric": METRIC, "value": v, "unit": info["unit"], "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "impl": "reference",
                "config": {"workload": describe(args.workload, args)}, "data": "synthetic",
                "cpu_baseline": {**info, "value": v},
                "e2e": {"value": v, "unit": info["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference has no CPU implementation of this path (its FP64 oracle is qiskit_aer, "
                        "not installed, and its CUDA extension is not a CPU path): the FP64 CPU restatement "
                        "named in cpu_baseline.sample stands in"}
        print(json.dumps(line))
        return 0

    import torch
    dev = local if torch.cuda.is_available() else 0
    torch.cuda.set_device(dev)
    dist_init(ws, "nccl")
    if args.jit < 0 and args.workload == "layers32":
        args.jit = 2   # specialise every pass before the timed region
    if args.jit >= 0:
        from qsim_b200 import engine as E
        E.set_jit(args.jit, 0, dev)
    if args.tile_bits or args.block_bits:
        from qsim_b200 import engine as E
        E._h(dev).call("qs_set_tile_bits", int(args.tile_bits))
        E._h(dev).call("qs_set_block_bits", int(args.block_bits))
    res, meta = WORKLOADS[args.workload](args, dev)
    # one config dict for both arms: the workload string; our arm's plan
    # details beside it
    cfg = res.pop("config", {})
    res["config"] = {"workload": cfg.get("workload", describe(args.workload, args))}
    if len(cfg) > 1:
        res["workload_details"] = {k: v for k, v in cfg.items() if k != "workload"}
    if args.workload == "layers32" and ws == 1 and not args.no_sub:
        res.update(headline_sub_records(args, dev))
    if rank == 0:
        res.update({"n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "data": "synthetic (seeded numpy PCG64)"})
        if ws == 1 and not args.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline(args.workload, args)
        print(json.dumps(res))
    barrier()
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
