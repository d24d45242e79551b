"""Regenerates ties.json: small graphs on which batch peeling meets the SAME density in two different rounds, so the
strict improvement rule (peel_improves, densest.h:76-78: a later round replaces the best only when strictly denser)
decides best_round. The four generated fixtures never tie, so these graphs pin that rule.

The graphs are found by a seeded search over small Erdos-Renyi graphs, using the oracle with the rule relaxed to
">=" as the detector (a graph qualifies when the relaxed rule changes the result). The EXPECTED outputs stored for
each graph come from the reference's own CPU code compiled from its headers (oracle/_ref/libga_ref.so): batch
peeling for every eps listed and the core decomposition (Alg 3 core numbers, level rounds).

Usage: ``python tests/golden/make_ties.py`` (needs the reference tree for oracle/_ref; the output is committed).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import Oracle, Reference  # noqa: E402

EPS = [(1, 10), (0, 1), (1, 1), (1, 2)]
WANT = 8


def _relaxed_oracle(tmp: str) -> Oracle:
    src = open(os.path.join(ROOT, "oracle", "ga_oracle.c")).read()
    old = "T * best_den > best_num * nalive"
    assert src.count(old) == 1
    path = os.path.join(tmp, "relaxed.c")
    open(path, "w").write(src.replace(old, "T * best_den >= best_num * nalive"))
    lib = os.path.join(tmp, "relaxed.so")
    subprocess.check_call(["gcc", "-O1", "-std=c11", "-fopenmp", "-fPIC", "-shared", "-I",
                           os.path.join(ROOT, "oracle"), path, "-o", lib])
    return Oracle(lib)


def main() -> None:
    ref, orc = Reference(), Oracle()
    rng = np.random.default_rng(2026)
    out = []
    with tempfile.TemporaryDirectory() as tmp:
        relaxed = _relaxed_oracle(tmp)
        while len(out) < WANT:
            n = int(rng.integers(6, 24))
            iu, iv = np.triu_indices(n, 1)
            keep = rng.random(iu.size) < float(rng.choice([0.2, 0.3, 0.5]))
            pairs = np.stack([iu[keep], iv[keep]], 1).astype(np.uint32)
            g = ref.build_graph_from_edges(n, orc.canonical_edges(pairs))
            tie = any((a.best_num, a.best_den, a.best_round) != (b.best_num, b.best_den, b.best_round)
                      for a, b in ((orc.batch_peel(g, num, den), relaxed.batch_peel(g, num, den)) for num, den in EPS))
            if not tie:
                continue
            peel = {}
            for num, den in EPS:
                r = ref.batch_peel(g, num, den)
                peel[f"{num}/{den}"] = {"best_num": r.best_num, "best_den": r.best_den, "best_round": r.best_round,
                                        "rounds": r.rounds, "removed_round": r.removed_round.tolist()}
            core, kmax, rounds = ref.core_levels(g)
            out.append({"n": n, "pairs": orc.canonical_edges(pairs).tolist(), "triangles": ref.triangles_serial(g),
                        "peel": peel, "core": core.tolist(), "kmax": kmax, "core_rounds": rounds})
    with open(os.path.join(HERE, "ties.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_ties.py (seed 2026)", "graphs": out}, f)
    print(f"wrote {len(out)} graphs")


if __name__ == "__main__":
    main()
