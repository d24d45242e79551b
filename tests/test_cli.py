"""The command-line drivers (ga_tc, ga_densest, ga_dsg), the replacements of the reference's gpu_tc / gpu_densest /
gpu_dsg: built against the C ABI, same usage and CSV columns; on a GPU their rows carry the oracle's numbers for the
golden fixtures."""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import FIXTURES, ROOT, fixture_path

BIN = os.path.join(ROOT, "graph_analyzer_b200", "_bin")
COLUMNS = {
    "ga_tc": "impl,graph,n,m,triangles,kernel_ms,h2d_ms,gpu_total_ms",                         # gpu_tc.cu:14-15
    "ga_densest": "impl,graph,n,m,best_triangles,best_vertices,density,rounds,time_ms,h2d_ms,total_ms",  # gpu_densest.cu:17
    "ga_dsg": "impl,graph,n,m,triangles,vertices,density,time_ms,h2d_ms,total_ms,rounds,kmax",  # gpu_dsg.cu:27
}


def _run(name, *args, timeout=300):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.fail(f"{exe} is not built (python -m graph_analyzer_b200.build)")
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=timeout)


def _rows(name, out):
    cols = COLUMNS[name].split(",")
    rows = []
    for line in out.strip().splitlines():
        f = line.split(",")
        assert len(f) == len(cols), line
        rows.append(dict(zip(cols, f)))
    return rows


@pytest.mark.parametrize("name", list(COLUMNS))
def test_usage(name):
    r = _run(name)
    assert r.returncode == 2 and "usage:" in r.stderr


@pytest.mark.parametrize("name", list(COLUMNS))
def test_no_device_fails_loudly(ga, name):
    if ga.device_count() > 0:
        pytest.skip("a GPU is present")
    r = _run(name, fixture_path("t_er300"), "--no-burnin")
    assert r.returncode == 1 and "GA_ERR_NO_DEVICE" in r.stderr and r.stdout == ""


def test_missing_file():
    r = _run("ga_tc", os.path.join(ROOT, "no_such_graph.txt"), "--no-burnin")
    assert r.returncode == 1 and r.stdout == ""


@pytest.mark.gpu
@pytest.mark.parametrize("fx", FIXTURES)
def test_ga_tc_rows(golden, cuda_ok, fx):
    r = _run("ga_tc", fixture_path(fx), "3", "--no-burnin")
    assert r.returncode == 0, r.stderr
    rows = _rows("ga_tc", r.stdout)
    assert [x["impl"] for x in rows] == ["gpu_hash_binned", "gpu_edge_per_thread", "gpu_autotuned"]
    for x in rows:
        assert int(x["triangles"]) == golden[fx]["triangles"]
        assert int(x["n"]) == golden[fx]["n"] and int(x["m"]) == golden[fx]["m"]
    r = _run("ga_tc", fixture_path(fx), "2", "--no-burnin", "--pinned")
    assert r.returncode == 0, r.stderr
    assert all(x["impl"].endswith("_pinned") for x in _rows("ga_tc", r.stdout))


def test_binary_csr_input_reaches_the_device_step(ga, tmp_path):
    """A .gacsr path is read by the binary loader (on a machine without a GPU the run then stops at the device)."""
    p = str(tmp_path / "g.gacsr")
    ga.save_csr(ga.load_graph(fixture_path("t_er300")), p)
    r = _run("ga_tc", p, "--no-burnin")
    assert "loaded n=300 m=2314" in r.stderr
    if ga.device_count() == 0:
        assert r.returncode == 1 and "GA_ERR_NO_DEVICE" in r.stderr
    else:
        assert r.returncode == 0 and all(int(x["triangles"]) == 652 for x in _rows("ga_tc", r.stdout))


@pytest.mark.gpu
@pytest.mark.parametrize("fx", FIXTURES)
@pytest.mark.parametrize("eps", [(1, 10), (1, 2)])
def test_ga_densest_rows(ga, oracle, cuda_ok, fx, eps):
    r = _run("ga_densest", fixture_path(fx), str(eps[0]), str(eps[1]), "--no-burnin", "--repeats", "2")
    assert r.returncode == 0, r.stderr
    rows = _rows("ga_densest", r.stdout)
    assert [x["impl"] for x in rows] == ["gpu_batch_peel", "gpu_batch_peel_host", "greedy_peel"]
    g = ga.load_graph(fixture_path(fx))
    o = oracle.batch_peel(g, *eps)
    for x in rows[:2]:
        assert (int(x["best_triangles"]), int(x["best_vertices"]), int(x["rounds"])) == (o.best_num, o.best_den,
                                                                                         o.rounds)
    w = oracle.greedy_pp(g, 1)                                   # cpu_greedy_peel's best (densest.h:209-252)
    assert (int(rows[2]["best_triangles"]), int(rows[2]["best_vertices"]), int(rows[2]["rounds"])) == (
        w.tri, w.verts, g.n)
    assert "density ratio gpu/greedy" in r.stderr
    r = _run("ga_densest", fixture_path(fx), str(eps[0]), str(eps[1]), "--no-burnin", "--repeats", "1", "--no-greedy")
    assert [x["impl"] for x in _rows("ga_densest", r.stdout)] == ["gpu_batch_peel", "gpu_batch_peel_host"]


@pytest.mark.gpu
@pytest.mark.parametrize("fx", FIXTURES)
def test_ga_dsg_rows(ga, oracle, cuda_ok, fx):
    """Core rows against the oracle; the pipeline rows (greedy, prune, Greedy++, seeded CoreExact, the full-graph
    check) against the reference's outputs for the same stages (tests/golden/dsg.json)."""
    r = _run("ga_dsg", fixture_path(fx), "--no-burnin", "--repeats", "2", "--verify-full")
    assert r.returncode == 0, r.stderr
    rows = {x["impl"]: x for x in _rows("ga_dsg", r.stdout)}
    assert list(rows) == ["gpu_core_decomp", "gpu_core_decomp_host", "greedy", "prune_kcore", "greedy_pp_pruned",
                          "core_exact_pruned_seeded", "pipeline_gpu_core", "core_exact_full"]
    g = ga.load_graph(fixture_path(fx))
    core, kmax, rounds = oracle.core_levels(g)
    tri, verts = oracle.core_level_density(g, core, kmax)
    for name in ("gpu_core_decomp", "gpu_core_decomp_host"):
        x = rows[name]
        assert (int(x["kmax"]), int(x["rounds"])) == (kmax, rounds)
        assert (int(x["triangles"]), int(x["vertices"])) == (tri, verts)
        assert np.isclose(float(x["density"]), tri / verts if verts else 0.0, rtol=1e-6)
    with open(os.path.join(ROOT, "tests", "golden", "dsg.json")) as f:
        rec = {x["name"]: x for x in json.load(f)["graphs"]}[fx]
    p = rec["pipeline"]

    def tv(x):
        return int(x["triangles"]), int(x["vertices"])

    assert tv(rows["greedy"]) == (rec["greedy"]["tri"], rec["greedy"]["verts"])
    x = rows["prune_kcore"]
    assert (int(x["n"]), int(x["m"]), int(x["triangles"]), int(x["rounds"])) == (
        p["pruned_n"], p["pruned_m"], p["pruned_triangles"], p["k"])
    assert tv(rows["greedy_pp_pruned"]) == (p["greedy_pp"]["tri"], p["greedy_pp"]["verts"])
    ex = p["core_exact_seeded"]
    assert tv(rows["core_exact_pruned_seeded"]) + (int(rows["core_exact_pruned_seeded"]["rounds"]),) == (
        ex["tri"], ex["verts"], ex["flow_calls"])
    assert tv(rows["pipeline_gpu_core"]) == (ex["tri"], ex["verts"])
    full = rec["core_exact"]
    assert tv(rows["core_exact_full"]) + (int(rows["core_exact_full"]["rounds"]),) == (
        full["tri"], full["verts"], full["flow_calls"])
    # --no-exact stops after the pruning and Greedy++ (gpu_dsg.cu's flags)
    r = _run("ga_dsg", fixture_path(fx), "--no-burnin", "--repeats", "1", "--no-exact", "--T", "5")
    assert r.returncode == 0, r.stderr
    assert [x["impl"] for x in _rows("ga_dsg", r.stdout)] == ["gpu_core_decomp", "gpu_core_decomp_host", "greedy",
                                                              "prune_kcore", "greedy_pp_pruned"]
