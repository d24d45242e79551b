"""Full-size golden records of the reference's own CPU code (run where the reference tree is; the output is committed).

Every input here is regenerated bit for bit from its seed by the library's host generators (the same calls the GPU
tests and bench.py make), so the records pin the device results at the workloads' full sizes to the reference's own
functions (oracle/_ref/libga_ref.so, its headers compiled by oracle/build_oracle.py):

* Holme-Kim, n = 1,700,000, 6 or 7 edges per new vertex (mean 6.54), triad probability 0.3, seed 1:
  T (cpu_triangles_serial, graph.h:110) and cpu_batch_peel (densest.h:138-160) at eps 1/20, 1/10, 1/2: every
  PeelResult field and a SHA-256 of removed_round.
* R-MAT scale 22, (a, b, c) = (.57, .19, .19), 8.52 * 2^22 samples, seed 1: T, a SHA-256 of the per-edge supports
  (for_each_triangle, dsg.h:67-79) and of the core numbers of core_decomposition (DSD Alg 3, dsg.h:125-166) with kmax.
  The level-round count of core_decomp_loop_inc comes from the oracle's incremental restatement (or_core_levels_inc):
  the reference's own level loop recounts every triangle in each of its thousands of rounds, which is out of reach
  at this size; or_core_levels_inc is pinned to that loop on smaller graphs (tests/test_oracle.py).
* The 4,096-graph Holme-Kim batch (n log-uniform in [64, 262,144], mean degree U[4, 32], p U[0.1, 0.7], seed 1):
  per graph T and the cpu_batch_peel (eps 1/10) fields (fullsize_batch.npz) and one SHA-256 over the concatenated
  removed_round arrays.

Usage: ``python tests/golden/make_fullsize.py [hk|rmat|batch ...]`` (default: all; R-MAT's Alg 3 takes the longest).
Writes tests/golden/fullsize.json (merged per part) and tests/golden/fullsize_batch.npz.
"""
from __future__ import annotations

import concurrent.futures as cf
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from fullsize_inputs import BATCH, HK, RMAT, SEED, batch_graphs, hk_graph, rmat_graph, sha  # noqa: E402
from oracle import Oracle, Reference  # noqa: E402

OUT = os.path.join(HERE, "fullsize.json")
OUT_BATCH = os.path.join(HERE, "fullsize_batch.npz")
EPS = [(1, 20), (1, 10), (1, 2)]


def log(*a):
    print(*a, flush=True)


def make_hk(ref: Reference) -> dict:
    g = hk_graph()
    rec = {"config": HK | {"seed": SEED}, "n": g.n, "m": g.m, "triangles": ref.triangles_serial(g), "peel": {}}
    for num, den in EPS:
        t0 = time.time()
        p = ref.batch_peel(g, num, den)
        assert p.ok
        rec["peel"][f"{num}/{den}"] = dict(best_num=p.best_num, best_den=p.best_den, best_round=p.best_round,
                                           rounds=p.rounds, removed_round_sha256=sha(p.removed_round))
        log(f"hk peel {num}/{den}: {time.time() - t0:.1f} s")
    return rec


def make_rmat(ref: Reference, orc: Oracle) -> dict:
    g = rmat_graph()
    rec = {"config": {k: list(v) if isinstance(v, tuple) else v for k, v in RMAT.items()} | {"seed": SEED},
           "n": g.n, "m": g.m}
    t0 = time.time()
    T, sup = ref.edge_support(g)
    rec |= {"triangles": T, "edge_support_sha256": sha(sup)}
    log(f"rmat supports: {time.time() - t0:.1f} s")
    t0 = time.time()
    core_i, kmax_i, rounds = orc.core_levels_inc(g)
    log(f"rmat or_core_levels_inc: {time.time() - t0:.1f} s, kmax {kmax_i}, {rounds} rounds")
    t0 = time.time()
    core, kmax = ref.core_decomposition(g)
    log(f"rmat core_decomposition: {time.time() - t0:.1f} s")
    assert kmax == kmax_i and np.array_equal(core, core_i), "oracle level loop disagrees with Alg 3"
    rec |= {"kmax": kmax, "core_sha256": sha(core), "core_rounds": rounds,
            "core_rounds_source": "or_core_levels_inc (oracle restatement of core_decomp_loop_inc)"}
    return rec


def make_batch(ref: Reference) -> dict:
    b = batch_graphs()
    G = b.num_graphs
    T = np.zeros(G, np.uint64)
    fields = np.zeros((G, 4), np.uint64)
    rr = [None] * G

    def one(i):
        g = b.graph(i)
        p = ref.batch_peel(g, 1, 10)
        return i, ref.triangles_serial(g), p

    t0 = time.time()
    with cf.ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        for i, t, p in ex.map(one, range(G)):
            assert p.ok, i
            T[i] = t
            fields[i] = (p.best_num, p.best_den, p.best_round, p.rounds)
            rr[i] = p.removed_round
    log(f"batch: {G} graphs in {time.time() - t0:.1f} s")
    np.savez_compressed(OUT_BATCH, triangles=T, best_num=fields[:, 0], best_den=fields[:, 1],
                        best_round=fields[:, 2].astype(np.uint32), rounds=fields[:, 3].astype(np.uint32))
    return {"config": BATCH | {"seed": SEED, "eps": "1/10"}, "N": int(b.vtx_off[-1]), "M": int(b.edge_off[-1]),
            "triangles_total": int(T.sum()), "removed_round_sha256": sha(np.concatenate(rr)),
            "per_graph": os.path.basename(OUT_BATCH)}


def main() -> None:
    parts = sys.argv[1:] or ["hk", "rmat", "batch"]
    ref, orc = Reference(), Oracle()
    rec = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for part in parts:
        t0 = time.time()
        rec[part] = {"hk": lambda: make_hk(ref), "rmat": lambda: make_rmat(ref, orc), "batch": lambda: make_batch(ref)}[
            part]()
        log(f"{part}: {time.time() - t0:.1f} s")
        with open(OUT, "w") as f:
            json.dump(rec, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
