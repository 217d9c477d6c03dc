"""The multi-GPU form of the benchmark is replicas only: each rank runs its
own particle set, and the step time reported is the maximum over ranks. These
tests run that host logic as two ``gloo`` ranks on the CPU:

  * the timing reduction returns the maximum over ranks on every rank;
  * the reference arm launched as the driver launches it (torch.distributed.run,
    two processes, rendezvous on 127.0.0.1) prints one JSON line, from rank 0
    only, and every rank exits 0.
"""
import json
import os
import socket
import subprocess
import sys
from types import SimpleNamespace

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, _ = bench.dist_setup(SimpleNamespace(impl="reference"))
    try:
        t = bench.dist_max(1.5 * (rank + 1), w, "reference")
        bench.dist_barrier(w)
        q.put((r, w, t))
    finally:
        bench.dist_done(w)


def test_step_time_is_the_max_over_ranks():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 3.0), (1, 2, 3.0)], got


def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--cpu-n1", "8"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1
