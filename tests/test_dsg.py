"""Densest subgraph by triangle density (CPU): the host stages of Greedy / Greedy++, CoreExact, Exact and
prune_to_core against the golden vectors of the reference's own dsg.h functions (tests/golden/dsg.json, written by
make_dsg.py), on triangle lists and core numbers made here by the checkers. The device entry points that produce
those inputs on the GPU are tested against the same vectors in test_gpu_dsg.py."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, fixture_path

with open(os.path.join(GOLDEN, "dsg.json")) as _f:
    DSG = json.load(_f)["graphs"]
BY_NAME = {g["name"]: g for g in DSG}


def dsg_graph(ga, rec):
    """The graph of a golden record, built by the product's host builder."""
    if rec["name"] in FIXTURES:
        return ga.load_graph(fixture_path(rec["name"]))
    if "holme_kim" in rec:
        h = rec["holme_kim"]
        pairs = ga.gen_holme_kim(h["n"], h["m_lo"], h["m_hi"], h["p_hi"], h["triad_p"], seed=h["seed"])
        return ga.graph_from_pairs(h["n"], pairs)
    return ga.build_graph_from_edges(rec["n"], np.array(rec["pairs"], np.uint32).reshape(-1, 2))


def triangles_of(g) -> np.ndarray:
    """Every triangle once, in for_each_triangle's order (dsg.h:67-79): (src[e], col[e], common out-neighbour)."""
    out = []
    rp, col = g.rowptr, g.col
    for u in range(g.n):
        nu = col[rp[u]:rp[u + 1]]
        for v in nu:
            common = np.intersect1d(nu, col[rp[v]:rp[v + 1]], assume_unique=True)
            out.extend((u, int(v), int(w)) for w in common)
    return np.array(out, np.uint32).reshape(-1, 3)


def incidence_of(n: int, tris: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Per-vertex lists of the other two corners of every triangle through the vertex."""
    owner = tris.reshape(-1)
    others = np.stack([tris[:, [1, 2]], tris[:, [0, 2]], tris[:, [0, 1]]], 1).reshape(-1, 2)
    order = np.argsort(owner, kind="stable")
    ptr = np.zeros(n + 1, np.uint64)
    np.add.at(ptr, owner.astype(np.int64) + 1, 1)
    return np.cumsum(ptr).astype(np.uint64), np.ascontiguousarray(others[order], np.uint32).reshape(-1)


def check(res, want, flows: bool = False):
    assert (res.tri, res.verts) == (want["tri"], want["verts"])
    assert res.set.tolist() == want["set"]
    if flows:
        assert (res.flow_calls, res.components_searched, res.shrinks) == (
            want["flow_calls"], want["components_searched"], want["shrinks"])


@pytest.fixture(scope="module")
def prepared(ga, oracle):
    """(graph, triangles, incidence, core numbers) of every golden graph."""
    out = {}
    for rec in DSG:
        g = dsg_graph(ga, rec)
        assert (g.n, g.m) == (rec["n"], rec["m"])
        tris = triangles_of(g)
        assert len(tris) == rec["triangles"]
        core, kmax, _ = oracle.core_levels(g)
        assert kmax == rec["kmax"]
        out[rec["name"]] = (g, tris, incidence_of(g.n, tris), core)
    return out


@pytest.mark.parametrize("name", list(BY_NAME))
def test_host_greedy_matches_reference(ga, prepared, name):
    rec = BY_NAME[name]
    g, _, (ip, ie), core = prepared[name]
    check(ga.greedy_pp_host(g.n, core, ip, ie, 1), rec["greedy"])
    if rec["triangles"]:
        assert [rec["greedy"]["tri"], rec["greedy"]["verts"]] == rec["cpu_greedy_peel"]
    for T, want in rec["greedy_pp"].items():
        r = ga.greedy_pp_host(g.n, core, ip, ie, int(T))
        check(r, want)
        assert [list(p) for p in r.per_pass] == want["per_pass"]


@pytest.mark.parametrize("name", list(BY_NAME))
def test_host_core_exact_matches_reference(ga, prepared, name):
    rec = BY_NAME[name]
    g, tris, _, core = prepared[name]
    check(ga.core_exact_host(g, tris, core), rec["core_exact"], flows=True)
    check(ga.core_exact_host(g, tris, core, use_pruning12=False), rec["core_exact_nopr"], flows=True)
    w = rec["greedy_pp"]["10"]
    seed = ga.DsgResult(w["tri"], w["verts"], np.array(w["set"], np.uint32))
    check(ga.core_exact_host(g, tris, core, seed=seed), rec["core_exact_seeded"], flows=True)


@pytest.mark.parametrize("name", [n for n in BY_NAME if "exact" in BY_NAME[n]])
def test_host_exact_matches_reference(ga, prepared, name):
    g, tris, _, _ = prepared[name]
    check(ga.exact_densest_host(g.n, tris), BY_NAME[name]["exact"], flows=True)


@pytest.mark.parametrize("name", list(BY_NAME))
def test_pipeline_matches_reference(ga, oracle, prepared, name):
    """gpu_dsg's stages after the core numbers (gpu_dsg.cu:318-369): prune to the ceil(lb)-core, Greedy++ with 10
    passes on the pruned graph, CoreExact seeded with it."""
    rec, p = BY_NAME[name], BY_NAME[name]["pipeline"]
    g, _, _, core = prepared[name]
    gp, old, core_p = ga.prune_to_core(g, core, p["k"])
    assert (gp.n, gp.m, old.tolist()) == (p["pruned_n"], p["pruned_m"], p["old_id"])
    assert np.array_equal(core_p, core[old])
    tris = triangles_of(gp)
    assert len(tris) == p["pruned_triangles"]
    ip, ie = incidence_of(gp.n, tris)
    gpp = ga.greedy_pp_host(gp.n, core_p, ip, ie, 10)
    check(gpp, p["greedy_pp"])
    check(ga.core_exact_host(gp, tris, core_p, seed=gpp), p["core_exact_seeded"], flows=True)


def test_prune_to_core_matches_reference(ga, reference, oracle):
    for name in FIXTURES:
        g = ga.load_graph(fixture_path(name))
        core, kmax, _ = oracle.core_levels(g)
        for k in sorted({0, 1, 2, kmax // 2, kmax, kmax + 1}):
            gp, old, cp = ga.prune_to_core(g, core, k)
            rp, rold, rcp = reference.prune_to_core(reference.load_graph(fixture_path(name)), core, k)
            assert (gp.n, gp.m, gp.max_out_degree) == (rp.n, rp.m, rp.max_out_degree)
            assert np.array_equal(gp.rowptr, rp.rowptr) and np.array_equal(gp.col, rp.col)
            assert np.array_equal(old, rold) and np.array_equal(cp, rcp)


def test_golden_file_is_the_reference_output(reference):
    """The small golden graphs reproduce from the reference compiled here (skipped where it is not built)."""
    for rec in DSG[:12]:
        if "pairs" in rec:
            g = reference.build_graph_from_edges(rec["n"], np.array(rec["pairs"], np.uint32).reshape(-1, 2))
        else:
            g = reference.load_graph(fixture_path(rec["name"]))
        r = reference.greedy_pp(g, 10)
        check(r, rec["greedy_pp"]["10"])
        core, _ = reference.core_decomposition(g)
        check(reference.core_exact(g, core), rec["core_exact"], flows=True)


def test_host_refusals(ga, prepared):
    g, tris, (ip, ie), core = prepared["t_pl900"]
    rec = BY_NAME["t_pl900"]
    with pytest.raises(ga.GAError) as e:
        ga.greedy_pp_host(g.n, core, ip, ie, 0)
    assert e.value.name == "GA_ERR_INVALID_ARGUMENT"
    # core numbers that are not the graph's: the greedy order check refuses them
    bad = core.copy()
    bad[np.argmax(core)] += 1
    with pytest.raises(ga.GAError) as e:
        ga.greedy_pp_host(g.n, bad, ip, ie, 1)
    assert e.value.name == "GA_ERR_INVALID_ARGUMENT"
    # a seed whose claimed triangle count is wrong is refused (dsg.h:545-551)
    w = rec["greedy_pp"]["10"]
    for tri, s in ((w["tri"] + 1, w["set"]), (w["tri"], w["set"][:-1]), (w["tri"], w["set"][:-1] + [w["set"][0]])):
        seed = ga.DsgResult(tri, w["verts"], np.array(s, np.uint32))
        with pytest.raises(ga.GAError) as e:
            ga.core_exact_host(g, tris, core, seed=seed)
        assert e.value.name == "GA_ERR_INVALID_ARGUMENT"
    # triangles that are not three distinct vertices < n
    with pytest.raises(ga.GAError):
        ga.exact_densest_host(3, np.array([[0, 1, 3]], np.uint32))
    with pytest.raises(ga.GAError):
        ga.exact_densest_host(3, np.array([[0, 1, 1]], np.uint32))


@pytest.mark.parametrize("name", list(BY_NAME))
def test_oracle_greedy_pinned(oracle, ga, name):
    """The oracle's C restatement of greedy_pp (the checker of the larger GPU cases) against the golden vectors."""
    rec = BY_NAME[name]
    g = dsg_graph(ga, rec)
    check(oracle.greedy_pp(g, 1), rec["greedy"])
    for T, want in rec["greedy_pp"].items():
        r = oracle.greedy_pp(g, int(T))
        check(r, want)
        assert [list(p) for p in r.per_pass] == want["per_pass"]


@pytest.mark.parametrize("seed", range(4))
def test_host_greedy_high_levels_vs_oracle(ga, oracle, seed):
    """Graphs whose core levels reach past 64 (the levels' queue switches from key buckets to a heap there), with
    sparse low levels beside them; the host stage against the oracle's pinned greedy_pp."""
    from conftest import random_pairs
    rng = np.random.default_rng(seed)
    n_dense, n_sparse = 30 + 5 * seed, 200
    dense = random_pairs(rng, n_dense, 0.85)
    sparse = random_pairs(rng, n_sparse, 0.03) + n_dense
    bridge = np.stack([rng.integers(0, n_dense, 40), rng.integers(n_dense, n_dense + n_sparse, 40)], 1)
    g = ga.graph_from_pairs(n_dense + n_sparse, np.concatenate([dense, sparse, bridge]).astype(np.uint32))
    core, kmax, _ = oracle.core_levels(g)
    assert kmax >= 64
    tris = triangles_of(g)
    ip, ie = incidence_of(g.n, tris)
    for passes in (1, 2):
        got, want = ga.greedy_pp_host(g.n, core, ip, ie, passes), oracle.greedy_pp(g, passes)
        assert (got.tri, got.verts, got.set.tolist(), got.per_pass) == (want.tri, want.verts, want.set.tolist(),
                                                                        want.per_pass)


def test_prune_to_core_refusals(ga):
    g = ga.build_graph_from_edges(4, np.array([[0, 1], [1, 2], [0, 2], [2, 3]], np.uint32))
    core = np.array([1, 1, 1, 0], np.uint32)
    gp, old, cp = ga.prune_to_core(g, core, 1)
    assert (gp.n, gp.m, old.tolist(), cp.tolist()) == (3, 3, [0, 1, 2], [1, 1, 1])
    gp, old, _ = ga.prune_to_core(g, core, 2)                     # nothing kept
    assert (gp.n, gp.m, old.size) == (0, 0, 0)
    bad = ga.Graph(g.n, g.m, g.rowptr.copy(), g.col.copy(), g.src, g.max_out_degree)
    bad.col[0] = 9                                                # endpoint >= n
    with pytest.raises(ga.GAError) as e:
        ga.prune_to_core(bad, core, 1)
    assert e.value.name == "GA_ERR_INVALID_GRAPH"
    bad = ga.Graph(g.n, g.m, g.rowptr.copy(), g.col.copy(), g.src, g.max_out_degree)
    bad.rowptr[-1] = g.m - 1                                      # rowptr does not span the edges
    with pytest.raises(ga.GAError) as e:
        ga.prune_to_core(bad, core, 1)
    assert e.value.name == "GA_ERR_INVALID_GRAPH"


@pytest.mark.parametrize("seed", range(3))
def test_host_exact_is_the_brute_force_optimum(ga, oracle, seed):
    """Independent of any implementation: on tiny graphs Exact and CoreExact (with and without Pruning1/2, seeded
    with Greedy++) reach the optimum density over all vertex subsets, Greedy++ stays at or below it and Greedy reaches
    at least a third of it (densest.h:11-14's guarantee for the triangle peel)."""
    from test_tiny_bruteforce import _brute_force, _tiny_graphs
    for n, pairs in _tiny_graphs(25, 300 + seed):
        g = ga.build_graph_from_edges(n, ga.canonical_edges(pairs))
        (bn, bd), _ = _brute_force(n, pairs)
        tris = triangles_of(g)
        ip, ie = incidence_of(g.n, tris)
        core, _, _ = oracle.core_levels(g)
        gpp = ga.greedy_pp_host(g.n, core, ip, ie, 5)
        gr = ga.greedy_pp_host(g.n, core, ip, ie, 1)
        for r in (ga.exact_densest_host(g.n, tris), ga.core_exact_host(g, tris, core),
                  ga.core_exact_host(g, tris, core, use_pruning12=False), ga.core_exact_host(g, tris, core, seed=gpp)):
            assert r.tri * (bd or 1) == bn * (r.verts or 1) and (r.verts == 0) == (bn == 0)
            assert len(r.set) == r.verts
        assert gpp.tri * (bd or 1) <= bn * (gpp.verts or 1)
        assert 3 * gr.tri * (bd or 1) >= bn * (gr.verts or 1)


@pytest.mark.parametrize("seed", range(3))
def test_host_mid_graphs_against_reference(ga, oracle, reference, seed):
    """The reference's --mid check (Exact as the oracle of CoreExact) on seeded mid-size graphs, with the reference's
    own functions run beside (skipped where the reference is not built): same sets, same flow-call counts."""
    from conftest import random_pairs
    rng = np.random.default_rng(500 + seed)
    for n, p in ((40, 0.35), (80, 0.2), (120, 0.12)):
        pairs = random_pairs(rng, n, p)
        g = ga.build_graph_from_edges(n, ga.canonical_edges(pairs))
        rg = reference.build_graph_from_edges(n, ga.canonical_edges(pairs))
        tris = triangles_of(g)
        core, _, _ = oracle.core_levels(g)
        ex, ce = ga.exact_densest_host(g.n, tris), ga.core_exact_host(g, tris, core)
        assert ex.tri * ce.verts == ce.tri * ex.verts
        for ours, theirs in ((ex, reference.exact_densest(rg)), (ce, reference.core_exact(rg, core))):
            assert (ours.tri, ours.verts, ours.set.tolist(), ours.flow_calls) == (
                theirs.tri, theirs.verts, theirs.set.tolist(), theirs.flow_calls)
        ip, ie = incidence_of(g.n, tris)
        ours, theirs = ga.greedy_pp_host(g.n, core, ip, ie, 4), reference.greedy_pp(rg, 4)
        assert (ours.tri, ours.verts, ours.set.tolist()) == (theirs.tri, theirs.verts, theirs.set.tolist())
