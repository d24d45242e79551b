"""Pins the oracle (oracle/ga_oracle.c) before anything is checked against it.

1. Known answers: the brute-force triangle counts printed by the reference's own fixture generators
   (scripts/gen_test_graph.py, scripts/gen_powerlaw.py, arguments of scripts/test_emu.sh:16-19) and the outputs the
   reference's own CPU code produced on those graphs (tests/golden/*.npz, from tests/golden/make_golden.py).
2. The reference compiled here (oracle/_ref), function by function, on random graphs.
3. Independent brute force (adjacency matrix, all-subset cores) on tiny graphs, as in emu_densest.cpp:19-40 and
   emu_dsg.cpp:28-82.
"""
from __future__ import annotations

import itertools
import json
import os

import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, fixture_path, golden_arrays, hub_pairs, random_pairs

EPS = [(1, 10), (1, 1), (0, 1), (3, 7), (1, 20), (1, 2)]


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_golden_fixtures(oracle, golden, name):
    g = oracle.load_graph(fixture_path(name))
    gold = golden[name]
    arr = golden_arrays(name)
    assert (g.n, g.m, g.max_out_degree) == (gold["n"], gold["m"], gold["max_out_degree"])
    assert np.array_equal(g.rowptr, arr["rowptr"]) and np.array_equal(g.col, arr["col"])
    assert np.array_equal(g.src, arr["src"])
    # the reference generator's brute-force count
    assert oracle.triangles_serial(g) == gold["brute_force_triangles"] == gold["triangles"]
    assert oracle.triangles_omp(g) == gold["triangles"]
    T, sup = oracle.edge_support(g)
    assert T == gold["triangles"] and np.array_equal(sup, arr["sup"])
    T, deg = oracle.triangle_degrees(g)
    assert np.array_equal(deg, arr["deg"])
    core, kmax = oracle.core_decomposition(g)
    assert kmax == gold["kmax"] and np.array_equal(core, arr["core"])
    core2, kmax2, rounds = oracle.core_levels(g)
    assert np.array_equal(core2, arr["core"]) and kmax2 == kmax and rounds == gold["core_rounds"]
    assert list(oracle.core_level_density(g, core, kmax)) == gold["kmax_core_density"]
    for num, den in EPS:
        p = oracle.batch_peel(g, num, den)
        want = gold["peel"][f"{num}/{den}"]
        assert p.ok
        assert (p.best_num, p.best_den, p.best_round, p.rounds) == (
            want["best_num"], want["best_den"], want["best_round"], want["rounds"])
        assert np.array_equal(p.removed_round, arr[f"removed_round_{num}_{den}"])


def _random_graph(oracle, rng, n, p):
    pairs = oracle.canonical_edges(random_pairs(rng, n, p))
    return oracle.build_graph_from_edges(n, pairs)


@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_reference_random(oracle, reference, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(20, 160))
    p = float(rng.choice([0.05, 0.15, 0.4]))
    raw = random_pairs(rng, n, p)
    # duplicates in both orientations and a self loop, like gen_test_graph.py:21-23
    extra = raw[rng.random(len(raw)) < 0.3][:, ::-1]
    raw = np.concatenate([raw, extra, np.array([[3, 3]], np.uint32)])
    pairs = oracle.canonical_edges(raw)
    g = oracle.build_graph_from_edges(n, pairs)
    r = reference.build_graph_from_edges(n, pairs)
    assert g.max_out_degree == r.max_out_degree
    assert all(np.array_equal(getattr(g, f), getattr(r, f)) for f in ("rowptr", "col", "src"))
    assert oracle.triangles_serial(g) == reference.triangles_serial(r) == reference.triangles_omp(r)
    assert np.array_equal(oracle.edge_support(g)[1], reference.edge_support(r)[1])
    assert np.array_equal(oracle.triangle_degrees(g)[1], reference.triangle_degrees(r)[1])
    for pa in (1.0, 0.7, 0.3, 0.0):
        alive = (rng.random(n) < pa).astype(np.uint8)
        a = oracle.participation(g, alive)
        b = reference.participation(r, alive)
        c = reference.participation(r, alive, use_omp=True)
        assert a[0] == b[0] == c[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[1], c[1])
    for num, den in EPS:
        po, pr = oracle.batch_peel(g, num, den), reference.batch_peel(r, num, den)
        assert po.ok == pr.ok
        assert (po.best_num, po.best_den, po.best_round, po.rounds) == (pr.best_num, pr.best_den, pr.best_round,
                                                                          pr.rounds)
        assert np.array_equal(po.removed_round, pr.removed_round)
    co, ko = oracle.core_decomposition(g)
    cr, kr = reference.core_decomposition(r)
    assert ko == kr and np.array_equal(co, cr)
    cl, kl, rl = oracle.core_levels(g)
    cl2, kl2, rl2 = reference.core_levels(r)
    assert np.array_equal(cl, cr) and (kl, rl) == (kl2, rl2)
    ur, uc = oracle.undirected_csr(g)
    ur2, uc2 = reference.undirected_csr(r)
    assert np.array_equal(ur, ur2) and np.array_equal(uc, uc2)


def test_oracle_matches_reference_hubs(oracle, reference):
    rng = np.random.default_rng(20261010)
    for _ in range(12):
        n, raw = hub_pairs(rng, int(rng.integers(1, 4)), int(rng.integers(40, 101)), int(rng.integers(8, 16)))
        pairs = oracle.canonical_edges(raw)
        g = oracle.build_graph_from_edges(n, pairs)
        r = reference.build_graph_from_edges(n, pairs)
        assert np.array_equal(g.col, r.col)
        co, ko = oracle.core_decomposition(g)
        cr, kr = reference.core_decomposition(r)
        assert ko == kr and np.array_equal(co, cr)
        assert oracle.core_levels(g)[2] == reference.core_levels(r)[2]


def test_oracle_arith_helpers_match_reference(oracle, reference):
    cases = [(100, 10**6, 1, 10), (0, 0, 0, 1), (4_000_000, 10**8, 1, 10), (10, 2**32, 1, 10), (10, 5, 1, 0),
             (10, 5, 2**20 + 1, 10), (2**31, 2**31, 1, 2**20), (7, 123456789, 3, 7)]
    for c in cases:
        assert oracle.peel_arith_ok(*c) == reference.peel_arith_ok(*c)
    for c in [(5, 10, 0, 0), (5, 10, 1, 2), (1, 2, 1, 2), (3, 4, 1, 2), (0, 5, 0, 7)]:
        assert oracle.peel_improves(*c) == reference.peel_improves(*c)


def test_oracle_load_graph_matches_reference(oracle, reference, tmp_path):
    p = tmp_path / "g.txt"
    p.write_text("# comment\n% other comment\n\n1 2\n2\t1\n3 3\n4 7\nbad line\n7 4 extra\n  9 1\n0 5\n")
    g, r = oracle.load_graph(str(p)), reference.load_graph(str(p))
    assert (g.n, g.m) == (r.n, r.m) == (10, 4)
    assert np.array_equal(g.col, r.col) and np.array_equal(g.rowptr, r.rowptr)


def _brute_participation(n, edges, alive):
    adj = np.zeros((n, n), bool)
    for a, b in edges:
        adj[a, b] = adj[b, a] = True
    tri = np.zeros(n, np.uint32)
    T = 0
    for u, v, w in itertools.combinations(range(n), 3):
        if alive[u] and alive[v] and alive[w] and adj[u, v] and adj[u, w] and adj[v, w]:
            T += 1
            tri[[u, v, w]] += 1
    return T, tri


def _brute_cores(n, edges):
    """core[v] = max k such that v lies in a subgraph with minimum triangle degree >= k (emu_dsg.cpp:10-12, 28-64)."""
    best = np.zeros(n, np.int64)
    for mask in range(1, 1 << n):
        members = [v for v in range(n) if mask >> v & 1]
        alive = np.zeros(n, np.uint8)
        alive[members] = 1
        _, tri = _brute_participation(n, edges, alive)
        k = min(int(tri[v]) for v in members)
        for v in members:
            best[v] = max(best[v], k)
    return best.astype(np.uint32)


@pytest.mark.parametrize("seed", range(8))
def test_oracle_against_brute_force(oracle, seed):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(5, 10))
    raw = random_pairs(rng, n, float(rng.choice([0.3, 0.5, 0.8])))
    g = oracle.build_graph_from_edges(n, oracle.canonical_edges(raw))
    edges = [(int(g.src[e]), int(g.col[e])) for e in range(g.m)]
    alive = (rng.random(n) < 0.8).astype(np.uint8)
    T, tri = _brute_participation(n, edges, alive)
    T2, tri2 = oracle.participation(g, alive)
    assert T == T2 and np.array_equal(tri, tri2)
    core, _ = oracle.core_decomposition(g)
    assert np.array_equal(core, _brute_cores(n, edges))


def _ties():
    with open(os.path.join(GOLDEN, "ties.json")) as f:
        return json.load(f)["graphs"]


@pytest.mark.parametrize("i", range(8))
def test_oracle_matches_reference_on_density_ties(oracle, i):
    """ties.json: outputs of the reference's own code on graphs where peeling meets one density twice (the strict
    improvement rule of densest.h:76-78 decides best_round)."""
    t = _ties()[i]
    g = oracle.build_graph_from_edges(t["n"], np.array(t["pairs"], np.uint32).reshape(-1, 2))
    assert oracle.triangles_serial(g) == t["triangles"]
    for key, want in t["peel"].items():
        num, den = map(int, key.split("/"))
        r = oracle.batch_peel(g, num, den)
        assert (r.best_num, r.best_den, r.best_round, r.rounds) == (want["best_num"], want["best_den"],
                                                                    want["best_round"], want["rounds"])
        assert r.removed_round.tolist() == want["removed_round"]
    core, kmax, rounds = oracle.core_levels(g)
    assert (kmax, rounds, core.tolist()) == (t["kmax"], t["core_rounds"], t["core"])


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("eps", [(1, 10), (0, 1), (3, 7)])
def test_best_round_recomputed_from_removed_round(oracle, name, eps):
    """The oracle's PeelResult against what its own removed_round array implies (the reference's emulator check)."""
    from peel_check import best_from_removed_round
    g = oracle.load_graph(fixture_path(name))
    r = oracle.batch_peel(g, *eps)
    assert (r.best_num, r.best_den, r.best_round, r.rounds) == best_from_removed_round(g, r.removed_round)


def test_incremental_level_loop_matches_reference(oracle, reference):
    """or_core_levels_inc (core_decomp_loop_inc restated with listed triangles) against the reference's own level loop
    (core_decomp_loop with a recount per round) and Alg 3, on fixtures, hubs, random, Holme-Kim and R-MAT graphs;
    or_edge_support_omp against the reference's for_each_triangle supports."""
    rng = np.random.default_rng(7)
    graphs = [oracle.load_graph(fixture_path(name)) for name in FIXTURES]
    for _ in range(4):
        n, raw = hub_pairs(rng, int(rng.integers(1, 4)), int(rng.integers(40, 101)), int(rng.integers(8, 16)))
        graphs.append(oracle.build_graph_from_edges(n, oracle.canonical_edges(raw)))
    graphs.append(oracle.build_graph_from_edges(120, random_pairs(rng, 120, 0.2)))
    graphs.append(oracle.build_graph_from_edges(1, np.zeros((0, 2), np.uint32)))
    import graph_analyzer_b200 as ga
    graphs.append(ga.graph_from_pairs(20000, ga.gen_holme_kim(20000, 6, 7, 0.54, 0.4, seed=9)))
    graphs.append(ga.graph_from_pairs(1 << 11, ga.gen_rmat(11, 10 << 11, seed=2)))
    for g in graphs:
        r = reference.build_graph_from_edges(g.n, np.stack([g.src, g.col], 1)) if g.m else g
        core, kmax, rounds = oracle.core_levels_inc(g)
        cr, kr, rr = reference.core_levels(r)
        assert (kmax, rounds) == (kr, rr) and np.array_equal(core, cr)
        ca, ka = reference.core_decomposition(r)
        assert ka == kmax and np.array_equal(ca, core)
        T, sup = oracle.edge_support(g, use_omp=True)
        Tr, supr = reference.edge_support(r)
        assert T == Tr and np.array_equal(sup, supr)
