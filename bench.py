"""Benchmark driver (one JSON line on rank 0).

Workloads (--workload):
  layers32  (default) 32-qubit state (2^32 complex64 = 32 GiB), 20 layers of
            Haar U(2) on every qubit + CZ brickwork + a Toffoli every 5th
            layer (954 gates).  value = gates/s of the fused tile passes on a
            state resident in HBM; e2e = gates/s of the public call path
            (host op list -> plan upload -> passes -> 1024 shots -> host).
  qv_batch  4096 Quantum-Volume circuits, widths uniform in [10, 20], depth =
            width, per-circuit seeds; value = circuits/s of the batch engine.
  qv12      one 12-qubit, depth-12 QV circuit; value = circuits/s.

--impl reference times the CPU implementation of the same workload: the FP64
statevector restatement (oracle/sv64.c, OpenMP on all host cores) on a
bounded sample, scaled to the metric's unit.  It is the only other place this
file runs oracle/ code besides the cpu_baseline leg.

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

METRIC = json.load(open(os.path.join(ROOT, "BASELINE.json")))["metric"] if os.path.exists(
    os.path.join(ROOT, "BASELINE.json")) else "served circuits/s"


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
        "config": {"workload": f"layers32: {n} qubits (2^{n} complex64 = {(8 << n) >> 30} GiB), {layers} layers "
                               f"U(2)+CZ brickwork+Toffoli/5, {ngates} gates, seed 0",
                   "passes": P, "tile_bits": info["tile_bits"], "blocks": info["n_blocks"],
                   "fused_ops": info["n_ops_fused"], "specialised_passes": info["n_jit_passes"],
                   "l2": "state 32 GiB >> 126 MB L2 (no flush needed)"},
        "hbm_gbs": achieved,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": kernel, "peak_source": src,
                     "algorithmic_bytes_per_launch": algo_bytes / P},
        "e2e": {"value": ws * ngates / te, "unit": "gates/s", "h2d_bytes_per_step": plan_bytes,
                "d2h_bytes_per_step": shots * 8},
        "gpu_launches": int(launches // max(1, args.steps)) * args.steps,
        "clocks": clk.summary(),
    }
    return res, {"n": n, "ops": ops, "unit": "gates/s", "ngates": ngates}


def bench_qv_batch(args, dev):
    import numpy as np
    import torch
    from qsim_b200 import engine as E
    from qsim_b200 import workloads as W
    C = args.circuits
    widths, oo, ops, so = W.qv_batch(C, 10, 20, seed=1)
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
    # weight the sample to the full width distribution
    per_width = {}
    for (w, _), c in zip(plans, idx):
        per_width.setdefault(w, []).append(c)
    plain_cps = len(idx) / t_plain
    # e2e: host ops -> batch plan (FP64 fusion, H2D) -> run -> probabilities of
    # circuit 0 back to the host, every step
    ops_host = np.ascontiguousarray(ops)

    def e2e_step():
        b2 = E.BatchPlan(widths, oo, ops_host, so, dev)
        b2.execute(states)
        r = states[: 1 << int(widths[0])].cpu()
        del b2
        return r

    e2e_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ne = max(1, args.steps // 2)
    for _ in range(ne):
        e2e_step()
    torch.cuda.synchronize()
    te = reduce_max((time.perf_counter() - t0) / ne, f"cuda:{dev}")
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    res = {
        "metric": METRIC, "value": ws * C / per_step, "unit": "circuits/s", "ms_per_step": per_step * 1e3,
        "dtype": "c64 (fp32 FMA; fp64 host fusion)",
        "config": {"workload": f"qv_batch: {C} QV circuits, widths U[10,20], depth=width, seeds 1e6*1+i",
                   "launches_per_step": bp.info["n_launches"], "items": bp.info["n_items"],
                   "max_passes": bp.info["max_passes"], "l2": "6.2 GB of states >> L2"},
        "per_circuit_launches": {"value": plain_cps, "unit": "circuits/s",
                                 "sample": f"{len(idx)} random circuits of the batch, one plan per circuit"},
        "hbm_gbs": achieved,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "k_pass<5>", "peak_source": src},
        "e2e": {"value": ws * C / te, "unit": "circuits/s", "h2d_bytes_per_step": int(ops.nbytes),
                "d2h_bytes_per_step": 8 << int(widths[0])},
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
            "dtype": "c64", "config": {"workload": "qv12: 12 qubits, depth 12, seed 0 (72 U(4))"},
            "clocks": clk.summary(), "gpu_launches": args.steps}, {"unit": "circuits/s"}


WORKLOADS = {"layers32": bench_layers32, "qv_batch": bench_qv_batch, "qv12": bench_qv12}


# --------------------------------------------------------- CPU baseline
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
        n_s = 26
        ops = W.layers_ops(n_s, 20, seed=0)[:96]
        psi = np.empty(1 << n_s, dtype=np.complex128)
        O.lib().sv64_init(psi.ctypes.data, n_s)
        t0 = time.perf_counter()
        O.lib().sv64_apply_ops(psi.ctypes.data, n_s, np.ascontiguousarray(ops).ctypes.data, len(ops))
        dt = time.perf_counter() - t0
        per_gate_32 = dt / len(ops) * 2 ** (args.qubits - n_s)
        return {"value": 1.0 / per_gate_32, "unit": "gates/s", "cores": cores, "kind": "port",
                "sample": f"first {len(ops)} gates of the same generator at {n_s} qubits (FP64), "
                          f"time x 2^{args.qubits - n_s} (extrapolated to {args.qubits} qubits)"}
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
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile-bits", type=int, default=0, help="planner tile bits (10..14; 0 = library default)")
    ap.add_argument("--block-bits", type=int, default=0, help="register-block qubits (2..5; 0 = default)")
    ap.add_argument("--jit", type=int, default=-1,
                    help="pass specialisation: 0 off, 1 plans >= 26 qubits, 2 all (-1 = library default)")
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
                "config": {"workload": args.workload}, "data": "synthetic",
                "cpu_baseline": {**info, "value": v},
                "e2e": {"value": v, "unit": info["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "reference CPU path = FP64 statevector restatement (oracle/sv64.c); qiskit_aer is not "
                        "installed and the reference's CUDA extension needs torch headers (not buildable here)"}
        print(json.dumps(line))
        return 0

    import torch
    dev = local if torch.cuda.is_available() else 0
    torch.cuda.set_device(dev)
    dist_init(ws, "nccl")
    if args.jit >= 0:
        from qsim_b200 import engine as E
        E.set_jit(args.jit, 0, dev)
    if args.tile_bits or args.block_bits:
        from qsim_b200 import engine as E
        E._h(dev).call("qs_set_tile_bits", int(args.tile_bits))
        E._h(dev).call("qs_set_block_bits", int(args.block_bits))
    res, meta = WORKLOADS[args.workload](args, dev)
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
