"""Regenerates dsg.json: expected outputs of the reference's densest-subgraph algorithms (dsg.h: greedy, greedy_pp,
core_exact with and without Pruning1/2 and with a Greedy++ seed, exact_densest, prune_to_core; densest.h:
cpu_greedy_peel) and of the pipeline its gpu_dsg driver runs (gpu_dsg.cu:318-369: lower bound = max(kmax-core
density, greedy density), prune to the ceil(lb)-core, Greedy++ with 10 passes, CoreExact seeded with it).

Every expected value comes from the reference's own CPU code compiled from its headers (oracle/_ref/libga_ref.so).
The graphs: the four generated fixtures, the density-tie graphs of ties.json, small seeded random graphs, graphs
built to have several equally dense optimal subgraphs (disjoint or overlapping cliques), and the Holme-Kim graph
n = 8,298, m_v = 12, p = 0.5, seed 1 (regenerated from its seed by the tests, so only its results are stored).

Usage: ``python tests/golden/make_dsg.py`` (needs the reference tree for oracle/_ref; the output is committed).
"""
from __future__ import annotations

import itertools
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from conftest import FIXTURES, fixture_path  # noqa: E402
from oracle import Oracle, Reference  # noqa: E402

PASSES = (3, 10)
HK = {"n": 8298, "m_lo": 12, "m_hi": 12, "p_hi": 0.0, "triad_p": 0.5, "seed": 1}


def _res(r) -> dict:
    return {"tri": r.tri, "verts": r.verts, "set": r.set.tolist(), "flow_calls": r.flow_calls,
            "components_searched": r.components_searched, "shrinks": r.shrinks}


def _dens_gt(a, b) -> bool:
    a = a if a[1] else (0, 1)
    b = b if b[1] else (0, 1)
    return a[0] * b[1] > b[0] * a[1]


def record(ref: Reference, g, with_exact: bool) -> dict:
    out = {"n": g.n, "m": g.m, "triangles": ref.triangles_serial(g)}
    gr = ref.greedy_pp(g, 1)
    out["greedy"] = _res(gr)
    out["cpu_greedy_peel"] = list(ref.cpu_greedy_peel(g))
    out["greedy_pp"] = {}
    for T in PASSES:
        r = ref.greedy_pp(g, T)
        out["greedy_pp"][str(T)] = dict(_res(r), per_pass=[list(p) for p in r.per_pass])
    core, kmax = ref.core_decomposition(g)
    out["kmax"] = kmax
    out["core_exact"] = _res(ref.core_exact(g, core))
    out["core_exact_nopr"] = _res(ref.core_exact(g, core, use_pruning12=False))
    out["core_exact_seeded"] = _res(ref.core_exact(g, core, True, ref.greedy_pp(g, 10)))
    if with_exact:
        out["exact"] = _res(ref.exact_densest(g))
    # the gpu_dsg pipeline (gpu_dsg.cu:318-369)
    lb = ref.core_level_density(g, core, kmax)
    if _dens_gt((gr.tri, gr.verts), lb):
        lb = (gr.tri, gr.verts)
    k = (lb[0] + lb[1] - 1) // lb[1] if lb[1] else 0
    gp, old, core_p = ref.prune_to_core(g, core, k)
    gpp = ref.greedy_pp(gp, 10)
    ex = ref.core_exact(gp, core_p, True, gpp)
    out["pipeline"] = {"lb": list(lb), "k": k, "pruned_n": gp.n, "pruned_m": gp.m,
                       "pruned_triangles": ref.triangles_serial(gp), "old_id": old.tolist(),
                       "greedy_pp": _res(gpp), "core_exact_seeded": _res(ex)}
    return out


def _random_graphs(rng, count):
    out = []
    for _ in range(count):
        n = int(rng.integers(5, 15))
        p = float(rng.choice([0.3, 0.5, 0.7, 0.9]))
        pairs = [(a, b) for a, b in itertools.combinations(range(n), 2) if rng.random() < p]
        out.append((n, pairs))
    return out


def _clique(vs):
    return [(a, b) for a, b in itertools.combinations(vs, 2)]


def _tie_graphs():
    """Graphs with several optimal subgraphs of equal density."""
    out = []
    out.append((10, _clique(range(5)) + _clique(range(5, 10))))                               # two disjoint K5
    out.append((9, _clique(range(5)) + _clique(range(4, 9))))                                 # two K5 sharing a vertex
    out.append((16, _clique(range(5)) + _clique(range(5, 10)) + _clique(range(10, 15)) + [(4, 5), (9, 10), (14, 15)]))
    out.append((12, _clique([0, 2, 4, 6]) + _clique([1, 3, 5, 7]) + _clique([8, 9, 10, 11]) + [(6, 8)]))
    out.append((7, _clique(range(6))))                                                        # K6 and an isolated vertex
    out.append((6, [(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5)]))                          # two triangles
    out.append((5, [(0, 1), (1, 2), (2, 3)]))                                                  # no triangle
    return out


def main() -> None:
    import graph_analyzer_b200 as ga

    ref, orc = Reference(), Oracle()
    graphs = []
    for name in FIXTURES:
        g = ref.load_graph(fixture_path(name))
        graphs.append(dict(record(ref, g, True), name=name))
    with open(os.path.join(HERE, "ties.json")) as f:
        for i, t in enumerate(json.load(f)["graphs"]):
            g = ref.build_graph_from_edges(t["n"], np.array(t["pairs"], np.uint32).reshape(-1, 2))
            graphs.append(dict(record(ref, g, True), name=f"tie{i}", pairs=t["pairs"]))
    rng = np.random.default_rng(2027)
    for i, (n, pairs) in enumerate(_random_graphs(rng, 30) + _tie_graphs()):
        canon = orc.canonical_edges(np.array(pairs, np.uint32).reshape(-1, 2))
        g = ref.build_graph_from_edges(n, canon)
        graphs.append(dict(record(ref, g, True), name=f"small{i}", pairs=canon.tolist()))
    pairs = ga.canonical_edges(ga.gen_holme_kim(HK["n"], HK["m_lo"], HK["m_hi"], HK["p_hi"], HK["triad_p"],
                                                seed=HK["seed"]))
    g = ref.build_graph_from_edges(HK["n"], pairs)
    graphs.append(dict(record(ref, g, False), name="hk8298", holme_kim=HK))
    with open(os.path.join(HERE, "dsg.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_dsg.py", "graphs": graphs}, f, separators=(",", ":"))
    print(f"wrote {len(graphs)} graphs")


if __name__ == "__main__":
    main()
