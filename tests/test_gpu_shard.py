"""The sharded count across ranks (ga_tc_count_shard, bench.py --shard): every rank is its own process that builds
and prepares its own copy of the graph on the device, counts its shard r of N, and the partial counts are summed with
one all-reduce (gloo here, on the host). The sum must equal the oracle's count: the shards that independent builds
cut must partition the triangles, whatever order each build's in-lists came out in. The ranks run on cuda:0 as
separate processes; their kernels never wait on one another, only the host all-reduce joins them."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


GRAPHS = {
    "rmat16": lambda ga: ga.graph_from_pairs(1 << 16, ga.gen_rmat(16, 10 << 16, seed=11)),
    "hk": lambda ga: ga.graph_from_pairs(60000, ga.gen_holme_kim(60000, 6, 14, 0.3, 0.6, seed=12)),
}


def _rank_main(rank, world, port, graph, kernel, q):
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    import graph_analyzer_b200 as ga
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        g = GRAPHS[graph](ga)
        with ga.DeviceGraph(g, device=0) as d:
            if kernel:
                d.set_option(ga.OPT_TC_KERNEL, kernel)
            part = d.tc_count_shard(rank, world)
        t = torch.tensor([part], dtype=torch.int64)
        dist.all_reduce(t)
        q.put((rank, part, int(t.item())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("graph", list(GRAPHS))
@pytest.mark.parametrize("kernel", [0, 1])
def test_sharded_count_across_processes(ga, oracle, cuda_ok, world, graph, kernel):
    want = oracle.triangles_omp(GRAPHS[graph](ga))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, graph, kernel, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert all(total == want for _, _, total in res)
    assert sum(part for _, part, _ in res) == want
