"""Parity at the workloads' full sizes against the reference's own CPU code: the device results on the Holme-Kim
n = 1.70M graph (batch peeling at eps 1/20, 1/10, 1/2), the R-MAT scale 22 graph (triangle count, every per-edge
support, every core number, kmax and the level-round count) and the 4,096-graph Holme-Kim batch (every graph's count
and PeelResult, and its removed_round) must equal the records tests/golden/make_fullsize.py made with the reference's
functions (cpu_triangles_serial, cpu_batch_peel, for_each_triangle, core_decomposition) on the same seeded inputs.
Arrays are compared through SHA-256 digests of their bytes (the batch's per-graph fields element by element)."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

sys.path.insert(0, GOLDEN)
from fullsize_inputs import batch_graphs, hk_graph, rmat_graph, sha  # noqa: E402

pytestmark = pytest.mark.gpu

EPS = [(1, 20), (1, 10), (1, 2)]


@pytest.fixture(scope="module")
def records():
    with open(os.path.join(GOLDEN, "fullsize.json")) as f:
        return json.load(f)


# (GA_OPT_TC_KERNEL, GA_OPT_LOOP_MODE, GA_OPT_UPDATE_MODE): autotuned kernel with graph-captured rounds over the
# incidence lists, and the plain form (one thread per edge, host-driven rounds, re-enumeration updates)
ARMS = {"tuned": (0, 2, 2), "plain": (1, 1, 1)}


def _arm(ga, d, arm):
    for opt, v in zip((ga.OPT_TC_KERNEL, ga.OPT_LOOP_MODE, ga.OPT_UPDATE_MODE), ARMS[arm]):
        d.set_option(opt, v)


@pytest.mark.parametrize("arm", list(ARMS))
def test_holme_kim_1_7m_peel(ga, cuda_ok, records, arm):
    rec = records["hk"]
    g = hk_graph()
    assert (g.n, g.m) == (rec["n"], rec["m"])
    with ga.DeviceGraph(g) as d:
        _arm(ga, d, arm)
        assert d.tc_count() == rec["triangles"]
        for num, den in EPS:
            want = rec["peel"][f"{num}/{den}"]
            r = d.batch_peel(num, den)
            assert (r.best_num, r.best_den, r.best_round, r.rounds) == (
                want["best_num"], want["best_den"], want["best_round"], want["rounds"]), (num, den)
            assert sha(r.removed_round) == want["removed_round_sha256"], (num, den)


def test_rmat22_supports_and_cores(ga, cuda_ok, records):
    rec = records["rmat"]
    g = rmat_graph()
    assert (g.n, g.m) == (rec["n"], rec["m"])
    with ga.DeviceGraph(g) as d:
        assert d.tc_count() == rec["triangles"]
        T, sup = d.support_edges()
        assert T == rec["triangles"]
        assert sha(sup) == rec["edge_support_sha256"]
        c = d.core_decomposition()
        assert (c.kmax, c.rounds) == (rec["kmax"], rec["core_rounds"])
        assert sha(c.core) == rec["core_sha256"]


def test_batch_4096_graphs(ga, cuda_ok, records):
    rec = records["batch"]
    with np.load(os.path.join(GOLDEN, rec["per_graph"])) as z:
        want = {k: z[k] for k in z.files}
    b = batch_graphs()
    assert (int(b.vtx_off[-1]), int(b.edge_off[-1])) == (rec["N"], rec["M"])
    with ga.DeviceBatch(b) as db:
        r = db.tc_peel(1, 10)
    assert np.all(r.status == 0)
    assert np.array_equal(r.triangles, want["triangles"])
    assert np.array_equal(r.best_num, want["best_num"]) and np.array_equal(r.best_den, want["best_den"])
    assert np.array_equal(r.best_round, want["best_round"]) and np.array_equal(r.rounds, want["rounds"])
    assert sha(r.removed_round) == rec["removed_round_sha256"]
