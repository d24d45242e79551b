"""GPU parity of the device-resident loops: triangle-density batch peeling (every PeelResult field and the whole
removed_round array, densest.h:56-59) and the (k, triangle)-core decomposition (every core number, kmax and the
level-round count of core_decomp_loop, dsg.h:693-717), in both loop modes, against the oracle and the golden
outputs of the reference's own CPU code."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import FIXTURES, fixture_path, golden_arrays, hub_pairs, random_pairs

pytestmark = pytest.mark.gpu

EPS = [(1, 10), (1, 1), (0, 1), (3, 7), (1, 20), (1, 2)]
# (GA_OPT_LOOP_MODE, GA_OPT_UPDATE_MODE): CUDA-graph or host-driven rounds x incidence-list or re-enumeration updates
MODES = {"graph-lists": (2, 2), "graph-enum": (2, 1), "host-lists": (1, 2), "host-enum": (1, 1)}


def _set_mode(ga, d, mode):
    loop, update = MODES[mode]
    d.set_option(ga.OPT_LOOP_MODE, loop)
    d.set_option(ga.OPT_UPDATE_MODE, update)


def _peel_eq(ga, oracle, g, d, num, den):
    o = oracle.batch_peel(g, num, den)
    r = d.batch_peel(num, den)
    assert o.ok
    assert (r.best_num, r.best_den, r.best_round, r.rounds) == (o.best_num, o.best_den, o.best_round, o.rounds)
    assert np.array_equal(r.removed_round, o.removed_round)
    assert ga.density_value(r.best_num, r.best_den) == ga.density_value(o.best_num, o.best_den)


def _core_eq(oracle, g, d):
    core, kmax, rounds = oracle.core_levels(g)
    r = d.core_decomposition()
    assert r.kmax == kmax and r.rounds == rounds
    assert np.array_equal(r.core, core)


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("mode", list(MODES))
def test_fixtures_peel_and_cores(ga, oracle, golden, cuda_ok, name, mode):
    g = ga.load_graph(fixture_path(name))
    arr = golden_arrays(name)
    with ga.DeviceGraph(g) as d:
        _set_mode(ga, d, mode)
        for num, den in EPS:
            r = d.batch_peel(num, den)
            want = golden[name]["peel"][f"{num}/{den}"]
            assert (r.best_num, r.best_den, r.best_round, r.rounds) == (
                want["best_num"], want["best_den"], want["best_round"], want["rounds"])
            assert np.array_equal(r.removed_round, arr[f"removed_round_{num}_{den}"])
        c = d.core_decomposition()
        assert c.kmax == golden[name]["kmax"] and c.rounds == golden[name]["core_rounds"]
        assert np.array_equal(c.core, arr["core"])


@pytest.mark.parametrize("seed", range(5))
@pytest.mark.parametrize("mode", list(MODES))
def test_random_graphs(ga, oracle, cuda_ok, seed, mode):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(30, 600))
    g = ga.build_graph_from_edges(n, ga.canonical_edges(random_pairs(rng, n, float(rng.choice([0.03, 0.1, 0.3])))))
    with ga.DeviceGraph(g) as d:
        _set_mode(ga, d, mode)
        for num, den in EPS:
            _peel_eq(ga, oracle, g, d, num, den)
        _core_eq(oracle, g, d)


@pytest.mark.parametrize("mode", ["graph-lists", "graph-enum"])
def test_hubs_and_wide_frontiers(ga, oracle, cuda_ok, mode):
    """Hubs with up to 600 neighbours: frontier vertices of degree > 256 take the binary-search update path and
    split into several update items (the reference's --hub suite, emu_dsg.cpp:654-696, widened)."""
    rng = np.random.default_rng(20261010)
    for _ in range(6):
        n, raw = hub_pairs(rng, int(rng.integers(1, 4)), int(rng.integers(40, 600)), int(rng.integers(8, 40)))
        g = ga.build_graph_from_edges(n, ga.canonical_edges(raw))
        with ga.DeviceGraph(g) as d:
            _set_mode(ga, d, mode)
            for num, den in EPS[:3]:
                _peel_eq(ga, oracle, g, d, num, den)
            _core_eq(oracle, g, d)


@pytest.mark.parametrize("mode", ["graph-lists", "graph-enum"])
def test_clique_and_edge_cases(ga, oracle, cuda_ok, mode):
    n = 300
    iu, iv = np.triu_indices(n, 1)
    cases = [
        (n, np.stack([iu, iv], 1).astype(np.uint32)),               # one level, degree 299 > 256
        (1, np.zeros((0, 2), np.uint32)),
        (6, np.zeros((0, 2), np.uint32)),                            # no edges: one round, everything at 0
        (3, np.array([[0, 1], [1, 2], [0, 2]], np.uint32)),
        (5, np.array([[0, 1], [1, 2], [2, 3], [3, 4]], np.uint32)),
    ]
    for nn, p in cases:
        g = ga.build_graph_from_edges(nn, p)
        with ga.DeviceGraph(g) as d:
            _set_mode(ga, d, mode)
            for num, den in EPS:
                _peel_eq(ga, oracle, g, d, num, den)
            _core_eq(oracle, g, d)


def test_holme_kim_c1_peel_and_cores(ga, oracle, cuda_ok):
    g = ga.graph_from_pairs(8298, ga.gen_holme_kim(8298, 12, 12, 0.0, 0.5, seed=1))
    with ga.DeviceGraph(g) as d:
        for mode in MODES:
            _set_mode(ga, d, mode)
            for num, den in [(1, 10), (1, 20), (1, 2)]:
                _peel_eq(ga, oracle, g, d, num, den)
            _core_eq(oracle, g, d)


def test_peel_refusals(ga, cuda_ok):
    g = ga.build_graph_from_edges(3, np.array([[0, 1], [1, 2], [0, 2]], np.uint32))
    with ga.DeviceGraph(g) as d:
        with pytest.raises(ga.GAError) as e:
            d.batch_peel(1, 0)
        assert e.value.name == "GA_ERR_INVALID_ARGUMENT"
        with pytest.raises(ga.GAError):
            d.batch_peel((1 << 20) + 1, 10)


def test_round_cap_reports_error(ga, oracle, cuda_ok):
    rng = np.random.default_rng(5)
    g = ga.build_graph_from_edges(200, ga.canonical_edges(random_pairs(rng, 200, 0.2)))
    rounds = oracle.core_levels(g)[2]
    assert rounds > 2
    with ga.DeviceGraph(g) as d:
        for mode in MODES:
            _set_mode(ga, d, mode)
            d.set_option(ga.OPT_MAX_ROUNDS, 2)
            with pytest.raises(ga.GAError) as e:
                d.core_decomposition()
            assert e.value.name == "GA_ERR_ROUND_LIMIT"
            d.set_option(ga.OPT_MAX_ROUNDS, 0)
            _core_eq(oracle, g, d)


def test_lists_reused_across_calls(ga, oracle, cuda_ok):
    """The incidence lists are built once per graph; later peel and core calls start from their lengths."""
    g = ga.graph_from_pairs(3000, ga.gen_holme_kim(3000, 6, 7, 0.54, 0.5, seed=3))
    with ga.DeviceGraph(g) as d:
        d.set_option(ga.OPT_UPDATE_MODE, 2)
        b0 = d.device_bytes()
        _core_eq(oracle, g, d)
        b1 = d.device_bytes()
        assert b1 > b0                                           # lists allocated by the first loop call
        for num, den in EPS:
            _peel_eq(ga, oracle, g, d, num, den)
        _core_eq(oracle, g, d)
        assert d.device_bytes() == b1                            # and reused
        d.set_option(ga.OPT_UPDATE_MODE, 1)                      # switching frees them
        _core_eq(oracle, g, d)
        assert d.device_bytes() < b1


def _ties():
    import json
    import os

    from conftest import GOLDEN
    with open(os.path.join(GOLDEN, "ties.json")) as f:
        return json.load(f)["graphs"]


@pytest.mark.parametrize("mode", list(MODES))
def test_density_ties_match_reference(ga, cuda_ok, mode):
    """Graphs whose peeling meets one density in two rounds: best_round follows the strict improvement rule
    (densest.h:76-78); expected outputs are the reference's own (tests/golden/ties.json)."""
    for t in _ties():
        g = ga.build_graph_from_edges(t["n"], np.array(t["pairs"], np.uint32).reshape(-1, 2))
        with ga.DeviceGraph(g) as d:
            _set_mode(ga, d, mode)
            assert d.tc_count() == t["triangles"]
            for key, want in t["peel"].items():
                num, den = map(int, key.split("/"))
                r = d.batch_peel(num, den)
                assert (r.best_num, r.best_den, r.best_round, r.rounds) == (
                    want["best_num"], want["best_den"], want["best_round"], want["rounds"]), key
                assert r.removed_round.tolist() == want["removed_round"]
            c = d.core_decomposition()
            assert (c.kmax, c.rounds, c.core.tolist()) == (t["kmax"], t["core_rounds"], t["core"])


def test_density_ties_in_one_batch(ga, cuda_ok):
    ties = _ties()
    graphs = [ga.build_graph_from_edges(t["n"], np.array(t["pairs"], np.uint32).reshape(-1, 2)) for t in ties]
    b = ga.pack_batch(graphs)
    with ga.DeviceBatch(b) as db:
        for key in ties[0]["peel"]:
            num, den = map(int, key.split("/"))
            r = db.tc_peel(num, den)
            for i, t in enumerate(ties):
                want = t["peel"][key]
                got = r.result(b, i)
                assert (got.best_num, got.best_den, got.best_round, got.rounds) == (
                    want["best_num"], want["best_den"], want["best_round"], want["rounds"]), (i, key)
                assert got.removed_round.tolist() == want["removed_round"]


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("eps", [(1, 10), (0, 1), (3, 7)])
def test_gpu_best_round_recomputed_from_removed_round(ga, cuda_ok, name, eps):
    """The device loop's PeelResult against what its removed_round array alone implies (the reference's emulator
    check, emu_densest.cpp:44-54,153-166)."""
    from peel_check import best_from_removed_round
    g = ga.load_graph(fixture_path(name))
    with ga.DeviceGraph(g) as d:
        r = d.batch_peel(*eps)
    assert (r.best_num, r.best_den, r.best_round, r.rounds) == best_from_removed_round(g, r.removed_round)


@pytest.mark.parametrize("kernel", [1, 2])
def test_core_level_density_every_level(ga, oracle, golden, cuda_ok, kernel):
    """core_level_density (dsg.h:169-174) on the device, at every core level of a Holme-Kim and an R-MAT graph and
    the golden kmax-core of each fixture, for both count kernels."""
    for name in FIXTURES:
        g = ga.load_graph(fixture_path(name))
        with ga.DeviceGraph(g) as d:
            d.set_option(ga.OPT_TC_KERNEL, kernel)
            got = d.core_level_density(golden_arrays(name)["core"], golden[name]["kmax"])
            assert list(got) == golden[name]["kmax_core_density"]
    for g in (ga.graph_from_pairs(2000, ga.gen_holme_kim(2000, 5, 6, 0.5, 0.5, seed=3)),
              ga.graph_from_pairs(1 << 12, ga.gen_rmat(12, 10 << 12, seed=5))):
        core, kmax, _ = oracle.core_levels(g)
        with ga.DeviceGraph(g) as d:
            d.set_option(ga.OPT_TC_KERNEL, kernel)
            for k in sorted(set(core.tolist()) | {0, kmax + 1}):
                assert d.core_level_density(core, k) == oracle.core_level_density(g, core, k), k
