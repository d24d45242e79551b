"""Densest subgraph by triangle density on the GPU, through the C ABI: Greedy / Greedy++ (core numbers and level
triangle lists from the device), CoreExact and Exact (triangles listed on the device), and the gpu_dsg pipeline
(gpu_dsg.cu:318-369) against the reference's own outputs (tests/golden/dsg.json), plus larger graphs against the
oracle's restatement of greedy_pp."""
from __future__ import annotations

import numpy as np
import pytest

from test_dsg import BY_NAME, check, dsg_graph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(BY_NAME))
def test_gpu_greedy(ga, cuda_ok, name):
    rec = BY_NAME[name]
    with ga.DeviceGraph(dsg_graph(ga, rec)) as d:
        check(d.greedy_pp(1), rec["greedy"])
        for T, want in rec["greedy_pp"].items():
            r = d.greedy_pp(int(T))
            check(r, want)
            assert [list(p) for p in r.per_pass] == want["per_pass"]


@pytest.mark.parametrize("name", list(BY_NAME))
def test_gpu_core_exact(ga, oracle, cuda_ok, name):
    rec = BY_NAME[name]
    g = dsg_graph(ga, rec)
    core, _, _ = oracle.core_levels(g)
    w = rec["greedy_pp"]["10"]
    seed = ga.DsgResult(w["tri"], w["verts"], np.array(w["set"], np.uint32))
    with ga.DeviceGraph(g) as d:
        check(d.core_exact(), rec["core_exact"], flows=True)                    # core numbers from the device
        check(d.core_exact(core), rec["core_exact"], flows=True)
        check(d.core_exact(core, use_pruning12=False), rec["core_exact_nopr"], flows=True)
        check(d.core_exact(seed=seed), rec["core_exact_seeded"], flows=True)
        if "exact" in rec:
            check(d.exact_densest(), rec["exact"], flows=True)


def _dens_gt(a, b) -> bool:
    """dens_gt (dsg.h:40-46): den 0 compares as 0."""
    a = a if a[1] else (0, 1)
    b = b if b[1] else (0, 1)
    return a[0] * b[1] > b[0] * a[1]


@pytest.mark.parametrize("name", list(BY_NAME))
def test_gpu_pipeline(ga, cuda_ok, name):
    """The gpu_dsg stages: device cores, lower bound max(kmax-core density, greedy), prune, Greedy++ (10 passes) and
    seeded CoreExact on the pruned graph."""
    rec, p = BY_NAME[name], BY_NAME[name]["pipeline"]
    g = dsg_graph(ga, rec)
    with ga.DeviceGraph(g) as d:
        cr = d.core_decomposition()
        kcore = (cr.core >= cr.kmax).astype(np.uint8)
        lb = (d.participation(kcore)[0], int(kcore.sum())) if g.n else (0, 0)   # core_level_density, dsg.h:169-174
        gr = d.greedy_pp(1)
    if _dens_gt((gr.tri, gr.verts), lb):
        lb = (gr.tri, gr.verts)
    assert list(lb) == p["lb"]
    k = (lb[0] + lb[1] - 1) // lb[1] if lb[1] else 0
    gp, old, core_p = ga.prune_to_core(g, cr.core, k)
    assert (gp.n, gp.m, old.tolist()) == (p["pruned_n"], p["pruned_m"], p["old_id"])
    with ga.DeviceGraph(gp) as dp:
        gpp = dp.greedy_pp(10)
        check(gpp, p["greedy_pp"])
        check(dp.core_exact(core_p, seed=gpp), p["core_exact_seeded"], flows=True)


def test_gpu_greedy_with_enumeration_update(ga, oracle, cuda_ok):
    """GA_OPT_UPDATE_MODE 1 makes the loops enumerate instead of keeping lists; Greedy builds the lists anyway and
    the loops keep their choice."""
    rec = BY_NAME["t_pl900"]
    g = dsg_graph(ga, rec)
    core, kmax, rounds = oracle.core_levels(g)
    with ga.DeviceGraph(g) as d:
        d.set_option(ga.OPT_UPDATE_MODE, 1)
        check(d.greedy_pp(3), rec["greedy_pp"]["3"])
        r = d.core_decomposition()
        assert np.array_equal(r.core, core) and (r.kmax, r.rounds) == (kmax, rounds)
        check(d.core_exact(), rec["core_exact"], flows=True)


@pytest.mark.parametrize("case", ["hk200k", "rmat16", "hubs"])
def test_gpu_greedy_larger_vs_oracle(ga, oracle, cuda_ok, case):
    """Graphs beyond the golden set: the device Greedy / Greedy++ against the oracle's greedy_pp."""
    if case == "hk200k":
        g = ga.graph_from_pairs(200_000, ga.gen_holme_kim(200_000, 6, 7, 0.54, 0.3, seed=5))
    elif case == "rmat16":
        g = ga.graph_from_pairs(1 << 16, ga.gen_rmat(16, 8 * (1 << 16), seed=3))
    else:
        from conftest import hub_pairs
        n, pairs = hub_pairs(np.random.default_rng(11), 6, 3000, 40)
        g = ga.graph_from_pairs(n, pairs)
    with ga.DeviceGraph(g) as d:
        for passes in (1, 2):
            want = oracle.greedy_pp(g, passes)
            got = d.greedy_pp(passes)
            assert (got.tri, got.verts) == (want.tri, want.verts)
            assert np.array_equal(got.set, want.set)
            assert got.per_pass == want.per_pass


def test_gpu_dsg_refusals(ga, cuda_ok):
    """Refusals through the device entry points: no passes, a seed that is not a subgraph with the claimed count, core
    numbers of the wrong length; the graph stays usable after each."""
    rec = BY_NAME["t_pl400"]
    g = dsg_graph(ga, rec)
    w = rec["greedy_pp"]["10"]
    with ga.DeviceGraph(g) as d:
        with pytest.raises(ga.GAError) as e:
            d.greedy_pp(0)
        assert e.value.name == "GA_ERR_INVALID_ARGUMENT"
        bad = ga.DsgResult(w["tri"] + 1, w["verts"], np.array(w["set"], np.uint32))
        with pytest.raises(ga.GAError) as e:
            d.core_exact(seed=bad)
        assert e.value.name == "GA_ERR_INVALID_ARGUMENT"
        with pytest.raises(ValueError):
            d.core_exact(np.zeros(g.n - 1, np.uint32))
        check(d.greedy_pp(10), w)
        check(d.core_exact(), rec["core_exact"], flows=True)
    # an empty graph and a graph without triangles
    with ga.DeviceGraph(ga.build_graph_from_edges(0, np.zeros((0, 2), np.uint32))) as d:
        assert (d.greedy_pp(3).verts, d.core_exact().verts, d.exact_densest().verts) == (0, 0, 0)
    with ga.DeviceGraph(ga.build_graph_from_edges(4, np.array([[0, 1], [1, 2], [2, 3]], np.uint32))) as d:
        r = d.greedy_pp(2)
        assert (r.tri, r.verts, r.per_pass) == (0, 0, [(0, 0), (0, 0)])
        assert (d.core_exact().tri, d.exact_densest().tri) == (0, 0)


def test_gpu_core_numbers_reused_only_while_valid(ga, oracle, cuda_ok):
    """The densest stages start from the last core loop's numbers when nothing ran since, and recompute them after a
    peeling loop (which rewrites the same device array)."""
    rec = BY_NAME["t_er800"]
    g = dsg_graph(ga, rec)
    core, _, _ = oracle.core_levels(g)
    with ga.DeviceGraph(g) as d:
        assert np.array_equal(d.core_decomposition().core, core)
        check(d.greedy_pp(1), rec["greedy"])                        # reuses the loop's numbers
        d.batch_peel(1, 10)                                         # out[] now holds removed_round
        check(d.greedy_pp(3), rec["greedy_pp"]["3"])
        check(d.core_exact(), rec["core_exact"], flows=True)
        d.batch_peel(1, 2)
        check(d.core_exact(), rec["core_exact"], flows=True)
        assert np.array_equal(d.core_decomposition().core, core)


@pytest.mark.parametrize("seed", range(2))
def test_gpu_exact_is_the_brute_force_optimum(ga, cuda_ok, seed):
    """On tiny graphs the device entry points reach the optimum over all vertex subsets (Exact, CoreExact), Greedy++
    stays at or below it and Greedy reaches at least a third of it."""
    from test_tiny_bruteforce import _brute_force, _tiny_graphs
    for n, pairs in _tiny_graphs(20, 400 + seed):
        g = ga.build_graph_from_edges(n, ga.canonical_edges(pairs))
        (bn, bd), _ = _brute_force(n, pairs)
        with ga.DeviceGraph(g) as d:
            gpp, gr = d.greedy_pp(5), d.greedy_pp(1)
            for r in (d.exact_densest(), d.core_exact(), d.core_exact(use_pruning12=False), d.core_exact(seed=gpp)):
                assert r.tri * (bd or 1) == bn * (r.verts or 1) and (r.verts == 0) == (bn == 0)
        assert gpp.tri * (bd or 1) <= bn * (gpp.verts or 1)
        assert 3 * gr.tri * (bd or 1) >= bn * (gr.verts or 1)
