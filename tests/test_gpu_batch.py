"""GPU parity of batches: every graph of a packed batch, counted and peeled together (one count launch, one
device-resident peeling loop), gives exactly what the oracle gives for that graph alone - triangle count and every
PeelResult field including removed_round (densest.h:56-59)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import random_pairs

pytestmark = pytest.mark.gpu

EPS = [(1, 10), (1, 1), (0, 1), (1, 20), (1, 2)]
MODES = {"graph-lists": (2, 2), "graph-enum": (2, 1), "host-lists": (1, 2)}


def _mixed_batch(ga, seed):
    rng = np.random.default_rng(seed)
    gs = [ga.build_graph_from_edges(1, np.zeros((0, 2), np.uint32)),                      # a lone vertex
          ga.build_graph_from_edges(9, np.zeros((0, 2), np.uint32))]                      # no edges
    iu, iv = np.triu_indices(40, 1)
    gs.append(ga.build_graph_from_edges(40, np.stack([iu, iv], 1).astype(np.uint32)))   # a clique
    for _ in range(6):
        n = int(rng.integers(20, 400))
        gs.append(ga.build_graph_from_edges(n, ga.canonical_edges(random_pairs(rng, n, float(rng.choice([0.03, 0.2]))))))
    hk = ga.gen_holme_kim_batch(12, 64, 2500, 4.0, 20.0, 0.1, 0.7, seed=seed)
    gs += [hk.graph(i) for i in range(hk.num_graphs)]
    order = rng.permutation(len(gs))
    return [gs[i] for i in order]


@pytest.mark.parametrize("mode", list(MODES))
def test_batch_matches_oracle_per_graph(ga, oracle, cuda_ok, mode):
    graphs = _mixed_batch(ga, 3)
    b = ga.pack_batch(graphs)
    with ga.DeviceBatch(b) as d:
        loop, update = MODES[mode]
        d.set_option(ga.OPT_LOOP_MODE, loop)
        d.set_option(ga.OPT_UPDATE_MODE, update)
        T = d.tc()
        for i, g in enumerate(graphs):
            assert T[i] == oracle.triangles_serial(g), i
        for num, den in EPS:
            r = d.tc_peel(num, den)
            assert np.array_equal(r.triangles, T)
            assert np.all(r.status == 0)
            for i, g in enumerate(graphs):
                o = oracle.batch_peel(g, num, den)
                got = r.result(b, i)
                assert (got.best_num, got.best_den, got.best_round, got.rounds) == (
                    o.best_num, o.best_den, o.best_round, o.rounds), (i, num, den)
                assert np.array_equal(got.removed_round, o.removed_round), (i, num, den)


def test_batch_equals_single_graph_api(ga, cuda_ok):
    b = ga.gen_holme_kim_batch(30, 64, 20000, 4.0, 32.0, 0.1, 0.7, seed=11)
    with ga.DeviceBatch(b) as d:
        r = d.tc_peel(1, 10)
    for i in range(b.num_graphs):
        g = b.graph(i)
        with ga.DeviceGraph(g) as one:
            assert one.tc_count() == r.triangles[i]
            assert one.batch_peel(1, 10) == r.result(b, i)


def test_batch_rejects_bad_input(ga, cuda_ok):
    g = ga.build_graph_from_edges(4, np.array([[0, 1], [1, 2], [0, 2]], np.uint32))
    b = ga.pack_batch([g, g])
    b.col[0] = 7                                                # a local id beyond its graph
    with pytest.raises(ga.GAError) as e:
        ga.DeviceBatch(b)
    assert e.value.name == "GA_ERR_INVALID_GRAPH"
