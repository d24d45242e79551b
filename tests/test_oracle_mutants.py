"""Mutation checks of the oracle (CPU): each mutant is a copy of oracle/ga_oracle.c with one planted mistake of the
kind the reference's own mutation list targets (scripts/mutation_check.py: kernel `<=` -> `<`, level rule, orientation
flip, ...), compiled on the side. The golden vectors of the reference's fixtures must expose every mutant, and the
unmutated copy must match them: this is what makes the oracle a pinned checker rather than a second opinion. The
golden vectors are the four generated fixtures plus ties.json (graphs whose peeling meets one density twice, outputs
from the reference's own code). The greedy_pp restatement has its own mutants, exposed by dsg.json (the reference's
greedy / greedy_pp outputs on 49 graphs)."""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

from conftest import ROOT

ORACLE_C = os.path.join(ROOT, "oracle", "ga_oracle.c")

MUTANTS = {
    "peel_threshold_strict": ("* nalive * den <= rhs", "* nalive * den < rhs"),
    "peel_rhs_eps": ("const uint64_t rhs = 3ull * (den + num) * T;", "const uint64_t rhs = 3ull * (den + 2 * num) * T;"),
    "improve_not_strict": ("T * best_den > best_num * nalive", "T * best_den >= best_num * nalive"),
    "orientation_tie_flip": ("deg[a] < deg[b] : (a) < (b))", "deg[a] < deg[b] : (a) > (b))"),
    "core_level_may_drop": ("if (mn > k) k = mn;", "k = mn;"),
    "core_frontier_strict": ("if (alive[v] && tri[v] <= k)", "if (alive[v] && tri[v] < k)"),
    "dedup_dropped": ("if (i > 0 && key[i] == key[i - 1]) continue;", ""),
    "intersect_skips": ("else { c++; i++; j++; }", "else { c++; i += 2; j++; }"),
}

# Mutants of the oracle's greedy_pp restatement (dsg.h:189-249), checked against the densest-subgraph golden vectors
# (tests/golden/dsg.json, the reference's own greedy / greedy_pp outputs).
DSG_MUTANTS = {
    "greedy_improve_not_strict": ("if (dens_gt_u(t, nalive, bn, bd)) { bn = t;",
                                  "if (!dens_gt_u(bn, bd, t, nalive)) { bn = t;"),
    "greedy_load_not_accumulated": ("next_load[v] = load[v] + cur[v];", "next_load[v] = cur[v];"),
    "greedy_cut_off_by_one": ("improved = 1; cut = norder; }", "improved = 1; cut = norder + (norder < n - 1); }"),
    "greedy_best_order_kept": ("if (improved) { memcpy(best_order", "if (!improved) { memcpy(best_order"),
}

DSG_CHECK = r"""
import json, sys
import numpy as np
sys.path.insert(0, {root!r})
from oracle import Oracle
from conftest import GOLDEN, FIXTURES, fixture_path
o = Oracle({lib!r})
diff = []
for rec in json.load(open(GOLDEN + "/dsg.json"))["graphs"]:
    if rec["name"] == "hk8298":
        continue
    if rec["name"] in FIXTURES:
        g = o.load_graph(fixture_path(rec["name"]))
    else:
        g = o.build_graph_from_edges(rec["n"], np.array(rec["pairs"], np.uint32).reshape(-1, 2))
    for T, want in [("1", rec["greedy"])] + list(rec["greedy_pp"].items()):
        r = o.greedy_pp(g, int(T))
        if (r.tri, r.verts, r.set.tolist()) != (want["tri"], want["verts"], want["set"]):
            diff.append((rec["name"], T))
print(diff)
sys.exit(3 if diff else 0)
"""

# Compares one compiled oracle with the golden vectors; exit 0 = all equal, 3 = a difference was found.
CHECK = r"""
import json, sys
import numpy as np
sys.path.insert(0, {root!r})
from oracle import Oracle
from conftest import FIXTURES, GOLDEN, fixture_path, golden_arrays
o = Oracle({lib!r})
gold = json.load(open(GOLDEN + "/golden.json"))
diff = []
for name in FIXTURES:
    g = o.load_graph(fixture_path(name))
    a, w = golden_arrays(name), gold[name]
    if (g.n, g.m) != (w["n"], w["m"]) or not np.array_equal(g.rowptr, a["rowptr"]) or not np.array_equal(g.col, a["col"]):
        diff.append((name, "csr")); continue
    if o.triangles_serial(g) != w["triangles"]:
        diff.append((name, "triangles"))
    for key, want in w["peel"].items():
        num, den = map(int, key.split("/"))
        r = o.batch_peel(g, num, den)
        if (r.best_num, r.best_den, r.best_round, r.rounds) != (want["best_num"], want["best_den"],
                want["best_round"], want["rounds"]) or not np.array_equal(r.removed_round, a[f"removed_round_{{num}}_{{den}}"]):
            diff.append((name, "peel", key))
    core, kmax, rounds = o.core_levels(g)
    if kmax != w["kmax"] or rounds != w["core_rounds"] or not np.array_equal(core, a["core"]):
        diff.append((name, "cores"))
for i, t in enumerate(json.load(open(GOLDEN + "/ties.json"))["graphs"]):   # density ties between rounds
    g = o.build_graph_from_edges(t["n"], np.array(t["pairs"], np.uint32).reshape(-1, 2))
    for key, want in t["peel"].items():
        num, den = map(int, key.split("/"))
        r = o.batch_peel(g, num, den)
        if (r.best_num, r.best_den, r.best_round, r.rounds) != (want["best_num"], want["best_den"],
                want["best_round"], want["rounds"]) or r.removed_round.tolist() != want["removed_round"]:
            diff.append(("tie", i, key))
    core, kmax, rounds = o.core_levels(g)
    if (kmax, rounds, core.tolist()) != (t["kmax"], t["core_rounds"], t["core"]):
        diff.append(("tie", i, "cores"))
print(diff)
sys.exit(3 if diff else 0)
"""


def _compile(tmp_path, name, text):
    src = tmp_path / f"{name}.c"
    src.write_text(text)
    lib = tmp_path / f"{name}.so"
    subprocess.check_call(["gcc", "-O1", "-std=c11", "-fopenmp", "-fPIC", "-shared", "-I",
                           os.path.join(ROOT, "oracle"), str(src), "-o", str(lib)])
    return str(lib)


def _check(lib, timeout=15, script=CHECK):
    """Exit status of the golden comparison; a mutant that never finishes (a loop that stops making progress) is
    stopped after `timeout` seconds and counts as exposed (status -1)."""
    code = script.format(root=ROOT, lib=lib)
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "tests"))
    try:
        return subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=timeout, env=env)
    except subprocess.TimeoutExpired:
        return subprocess.CompletedProcess([], -1, "", "timed out")


def test_unmutated_copy_matches_golden(tmp_path):
    lib = _compile(tmp_path, "clean", open(ORACLE_C).read())
    r = _check(lib, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    r = _check(lib, timeout=300, script=DSG_CHECK)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.parametrize("mutant", list(MUTANTS))
def test_golden_vectors_kill_mutant(tmp_path, mutant):
    old, new = MUTANTS[mutant]
    text = open(ORACLE_C).read()
    assert text.count(old) == 1, f"mutation site of {mutant} not found exactly once"
    r = _check(_compile(tmp_path, mutant, text.replace(old, new)))
    # killed: a golden mismatch (exit 3) or the mutant failing outright (crash, exception)
    assert r.returncode != 0, f"mutant {mutant} survived the golden vectors"


@pytest.mark.parametrize("mutant", list(DSG_MUTANTS))
def test_dsg_golden_vectors_kill_mutant(tmp_path, mutant):
    old, new = DSG_MUTANTS[mutant]
    text = open(ORACLE_C).read()
    assert text.count(old) == 1, f"mutation site of {mutant} not found exactly once"
    r = _check(_compile(tmp_path, mutant, text.replace(old, new)), script=DSG_CHECK)
    assert r.returncode != 0, f"mutant {mutant} survived the golden vectors"
