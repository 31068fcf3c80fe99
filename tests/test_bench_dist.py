"""bench.py's multi-rank plumbing on CPU: world_size-2 gloo ranks (barrier,
max-over-ranks timing) and the reference arm's rank-0-only rule."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    bench.dist_init(ws, "gloo")
    bench.barrier()
    m = bench.reduce_max(1.5 + rank)
    bench.barrier()
    q.put((rank, m))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 2.5, 1: 2.5}


def test_reference_arm_only_rank0_prints():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "qv12",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "qv12",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_units_match_each_workload():
    """The reference arm reports each workload in its metric's unit (the
    driver divides the two arms' values), here on quick variants."""
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    for wl, extra, unit in (("serving", ["--requests", "20"], "requests/s"),
                            ("adjoint", ["--qubits", "10"], "gradients/s"),
                            ("chebyshev", ["--qubits", "12"], "evolutions/s"),
                            ("noisy", ["--qubits", "6"], "trajectories/s")):
        r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", wl,
                            "--steps", "1", "--warmup", "0", *extra], env=env, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr
        line = json.loads(r.stdout.strip().splitlines()[-1])
        assert line["unit"] == unit and line["cpu_baseline"]["unit"] == unit and line["value"] > 0, line


def test_reference_arm_config_is_the_shared_workload_string():
    """Both arms print config = {"workload": describe(...)}, so the two lines
    name the same workload."""
    import argparse
    sys.path.insert(0, ROOT)
    import bench
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "qv12",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    ns = argparse.Namespace(qubits=32, circuits=4096, requests=200, rates="50,100,200,500,1000,2000", workers=4,
                            server="native")
    assert line["config"] == {"workload": bench.describe("qv12", ns)}
    assert bench.describe("layers32", ns).startswith("layers32: 32 qubits") and "954 gates" in \
        bench.describe("layers32", ns)
