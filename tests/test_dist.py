"""The multi-rank host logic of bench.py on CPU (gloo, world size 2): the max-over-ranks timing reduction, and the
reference arm under torchrun, where rank 0 alone runs and prints one line and the other rank exits 0 without work.
The GPU arm shares dist_setup / max_over_ranks; its ranks are replicas with no collective on the data path."""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    got = bench.max_over_ranks(dist, 10.0 * rank + 0.5)
    dist.destroy_process_group()
    q.put((rank, got))


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 10.5, 1: 10.5}


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.25) == 3.25


def test_reference_arm_two_ranks(reference):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--gpus", "2", "--scale", "10", "--steps", "2", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["steps"] == 2
    assert line["config"]["workload"] == "rmat10_tc" and line["config"]["triangles"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
