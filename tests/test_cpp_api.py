"""The reference-names C++ surface (include/ga/graph_analyzer.hpp: Graph, load_graph, PeelResult, batch_peel_loop,
core_decomp_loop_inc, greedy / greedy_pp / prune_to_core / core_exact) compiled into a small program as a maintainer of the reference would, linked against the
library; on a GPU its results must equal the golden outputs of the reference's own code."""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, ROOT, fixture_path, golden_arrays

LIB_DIR = os.path.join(ROOT, "graph_analyzer_b200", "_lib")


@pytest.fixture(scope="module")
def api_check(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "api_check")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "api_check.cpp"), "-o", exe, "-L", LIB_DIR,
                           "-lga_b200", f"-Wl,-rpath,{LIB_DIR}"])
    return exe


def _hash(a):
    h = 0
    for x in a.tolist():
        h = (h * 1000003 + int(x)) & ((1 << 64) - 1)
    return format(h, "x")


def test_compiles_and_refuses_bad_usage(api_check):
    assert subprocess.run([api_check], capture_output=True).returncode == 2


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_reference_names_match_golden(api_check, golden, cuda_ok, name):
    w, a = golden[name], golden_arrays(name)
    r = subprocess.run([api_check, fixture_path(name), "1", "10", str(w["triangles"])], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = dict(line.split(" ", 1) for line in r.stdout.strip().splitlines())
    assert int(out["triangles"]) == w["triangles"]
    p = w["peel"]["1/10"]
    assert out["peel"].split() == [str(p["best_num"]), str(p["best_den"]), str(p["best_round"]), str(p["rounds"]),
                                   _hash(a["removed_round_1_10"])]
    assert out["cores"].split() == [str(w["kmax"]), str(w["core_rounds"]), _hash(a["core"])]
    assert out["kcore"].split() == [str(x) for x in w["kmax_core_density"]]   # core_level_density, dsg.h:169
    assert out["supports"].split() == [str(w["triangles"])] * 2
    assert out["refusals"].split() == ["0", "0"]
    assert out["batch_serve"].split() == ["1", "1"]      # DeviceBatch and Server give the single-graph results
    with open(os.path.join(GOLDEN, "dsg.json")) as f:
        rec = {x["name"]: x for x in json.load(f)["graphs"]}[name]
    p = rec["pipeline"]
    assert out["dsg"].split() == [str(x) for x in (
        rec["greedy"]["tri"], rec["greedy"]["verts"], p["pruned_n"], p["pruned_m"], p["greedy_pp"]["tri"],
        p["greedy_pp"]["verts"], p["core_exact_seeded"]["tri"], p["core_exact_seeded"]["verts"],
        p["core_exact_seeded"]["flow_calls"])]
