"""The full-size records (tests/golden/fullsize.json, fullsize_batch.npz, written by make_fullsize.py from the
reference's own CPU code) hold together on CPU: the seeded inputs regenerate to the recorded sizes, and the oracle
reproduces the recorded Holme-Kim n = 1.70M peeling at eps 1/10, the R-MAT scale 22 triangle count and a sample of
the batch's graphs. The device results are compared with the same records in test_gpu_fullsize.py."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

sys.path.insert(0, GOLDEN)
from fullsize_inputs import batch_graphs, hk_graph, rmat_graph, sha  # noqa: E402


@pytest.fixture(scope="module")
def records():
    with open(os.path.join(GOLDEN, "fullsize.json")) as f:
        return json.load(f)


def test_holme_kim_record(oracle, records):
    rec = records["hk"]
    g = hk_graph()
    assert (g.n, g.m) == (rec["n"], rec["m"])
    assert oracle.triangles_omp(g) == rec["triangles"]
    r = oracle.batch_peel(g, 1, 10)
    want = rec["peel"]["1/10"]
    assert (r.best_num, r.best_den, r.best_round, r.rounds) == (want["best_num"], want["best_den"], want["best_round"],
                                                                want["rounds"])
    assert sha(r.removed_round) == want["removed_round_sha256"]


@pytest.mark.slow
def test_rmat_record_count(oracle, records):
    rec = records["rmat"]
    g = rmat_graph()
    assert (g.n, g.m) == (rec["n"], rec["m"])
    assert oracle.triangles_omp(g) == rec["triangles"]


def test_batch_record_sample(oracle, records):
    rec = records["batch"]
    with np.load(os.path.join(GOLDEN, rec["per_graph"])) as z:
        want = {k: z[k] for k in z.files}
    b = batch_graphs()
    assert (b.num_graphs, int(b.vtx_off[-1]), int(b.edge_off[-1])) == (rec["config"]["graphs"], rec["N"], rec["M"])
    assert int(want["triangles"].sum()) == rec["triangles_total"]
    sizes = np.diff(b.edge_off.astype(np.int64))
    sample = np.argsort(sizes)[:: max(1, b.num_graphs // 24)][:24]   # small to large
    for i in sample[sizes[sample] < 2_000_000]:
        g = b.graph(int(i))
        r = oracle.batch_peel(g, 1, 10)
        assert oracle.triangles_serial(g) == want["triangles"][i]
        assert (r.best_num, r.best_den, r.best_round, r.rounds) == (
            want["best_num"][i], want["best_den"][i], want["best_round"][i], want["rounds"][i])
