"""Brute force over every vertex subset of tiny graphs (the reference's --tiny checks, emu_densest.cpp:191-239 and
emu_dsg.cpp:28-64, restated as properties):
  * core numbers equal their definition: core[v] = the largest k such that some vertex set S containing v has every
    member in at least k triangles inside S (emu_dsg.cpp:10-12);
  * batch peeling returns a real subgraph density not above the optimum and within its 3(1 + eps) guarantee
    (densest.h:11-14).
Checked on the oracle (CPU) and on the GPU paths."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

EPS = [(1, 10), (0, 1), (1, 1), (1, 2)]


def _tiny_graphs(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(5, 12))
        p = float(rng.choice([0.3, 0.5, 0.7, 0.9]))
        pairs = [(a, b) for a, b in itertools.combinations(range(n), 2) if rng.random() < p]
        out.append((n, np.array(pairs, np.uint32).reshape(-1, 2)))
    return out


def _brute_force(n, pairs):
    """(optimum density as (num, den), definitional core numbers) over all 2^n vertex sets."""
    adj = np.zeros((n, n), bool)
    for a, b in pairs:
        adj[a, b] = adj[b, a] = True
    tris = [(a, b, c) for a, b, c in itertools.combinations(range(n), 3) if adj[a, b] and adj[a, c] and adj[b, c]]
    tmask = np.array([(1 << a) | (1 << b) | (1 << c) for a, b, c in tris], np.int64)
    corner = np.zeros((len(tris), n), bool)
    for i, t in enumerate(tris):
        corner[i, list(t)] = True
    best = (0, 0)
    core = np.zeros(n, np.int64)
    for S in range(1, 1 << n):
        inside = (tmask & S) == tmask if len(tris) else np.zeros(0, bool)
        T = int(inside.sum())
        size = bin(S).count("1")
        if T * (best[1] or 1) > best[0] * size or best[1] == 0 and T > 0:
            best = (T, size)
        members = [v for v in range(n) if S >> v & 1]
        per = corner[inside].sum(0) if len(tris) else np.zeros(n, np.int64)
        k = int(min(per[v] for v in members))
        for v in members:
            core[v] = max(core[v], k)
    return best, core


def _check_peel(best, num, den, r):
    opt_num, opt_den = best
    if opt_num == 0:
        assert r.best_num == 0
        return
    # the returned density is a real subgraph's: not above the optimum
    assert r.best_num * opt_den <= opt_num * r.best_den
    # guarantee: density >= opt / (3 (1 + eps))  <=>  best_num * 3 * (den + num) * opt_den >= opt_num * den * best_den
    assert r.best_num * 3 * (den + num) * opt_den >= opt_num * den * r.best_den


@pytest.mark.parametrize("seed", range(3))
def test_oracle_on_tiny_graphs(oracle, seed):
    for n, pairs in _tiny_graphs(25, seed):
        g = oracle.build_graph_from_edges(n, oracle.canonical_edges(pairs))
        best, core = _brute_force(n, pairs)
        c, _, _ = oracle.core_levels(g)
        assert np.array_equal(c, core)
        for num, den in EPS:
            _check_peel(best, num, den, oracle.batch_peel(g, num, den))


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(3))
def test_gpu_on_tiny_graphs(ga, cuda_ok, seed):
    graphs = _tiny_graphs(25, 100 + seed)
    hosts = [ga.build_graph_from_edges(n, ga.canonical_edges(pairs)) for n, pairs in graphs]
    truth = [_brute_force(n, pairs) for n, pairs in graphs]
    for g, (best, core) in zip(hosts, truth):
        with ga.DeviceGraph(g) as d:
            for loop in (1, 2):
                d.set_option(ga.OPT_LOOP_MODE, loop)
                assert np.array_equal(d.core_decomposition().core, core)
                for num, den in EPS:
                    _check_peel(best, num, den, d.batch_peel(num, den))
    # the same graphs peeled together as one batch
    b = ga.pack_batch(hosts)
    with ga.DeviceBatch(b) as db:
        for num, den in EPS:
            r = db.tc_peel(num, den)
            for i, (best, _) in enumerate(truth):
                _check_peel(best, num, den, r.result(b, i))
