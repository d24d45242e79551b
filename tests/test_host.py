"""Host side of the product (no GPU): the C-ABI library loads and exports every declared symbol, and the graph.h
surface (edge clean-up, (degree,id) orientation, CSR, text loader) and the generators behave like the reference."""
from __future__ import annotations

import os
import re

import numpy as np
import pytest

from conftest import FIXTURES, ROOT, fixture_path, golden_arrays, random_pairs


def _declared_symbols() -> set[str]:
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(ga_\w+)\s*\(", text, re.M))
    return names


def test_library_exports_every_declared_symbol(ga):
    declared = _declared_symbols()
    assert len(declared) >= 25
    L = ga.lib()
    missing = [s for s in sorted(declared) if not hasattr(L, s)]
    assert not missing, missing
    assert set(ga.SIGNATURES) <= declared


def test_status_strings(ga):
    L = ga.lib()
    for code, name in ga.STATUS.items():
        assert L.ga_status_string(code).decode() == name


@pytest.mark.parametrize("name", FIXTURES)
def test_load_graph_matches_reference_layout(ga, golden, name):
    g = ga.load_graph(fixture_path(name))
    arr = golden_arrays(name)
    assert g.n == golden[name]["n"] and g.m == golden[name]["m"]
    assert g.max_out_degree == golden[name]["max_out_degree"]
    assert np.array_equal(g.rowptr, arr["rowptr"]) and np.array_equal(g.col, arr["col"])
    assert np.array_equal(g.src, arr["src"])


@pytest.mark.parametrize("seed", range(5))
def test_build_graph_matches_oracle(ga, oracle, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 3000))
    raw = random_pairs(rng, min(n, 400), 0.05) if n < 400 else rng.integers(0, n, (6 * n, 2)).astype(np.uint32)
    # reversed duplicates and self loops must be cleaned exactly like load_graph (graph.h:85-92)
    raw = np.concatenate([raw, raw[: len(raw) // 3, ::-1], np.array([[1, 1]], np.uint32)])
    a = ga.canonical_edges(raw)
    b = oracle.canonical_edges(raw)
    assert np.array_equal(a, b)
    g = ga.build_graph_from_edges(n, a)
    o = oracle.build_graph_from_edges(n, b)
    assert (g.n, g.m, g.max_out_degree) == (o.n, o.m, o.max_out_degree)
    assert np.array_equal(g.rowptr, o.rowptr) and np.array_equal(g.col, o.col) and np.array_equal(g.src, o.src)
    assert ga.graph_from_pairs(n, raw) == g


def test_build_graph_rejects_bad_input(ga):
    with pytest.raises(ga.GAError) as e:
        ga.build_graph_from_edges(3, np.array([[0, 5]], np.uint32))
    assert e.value.name == "GA_ERR_INVALID_GRAPH"
    with pytest.raises(ga.GAError):
        ga.build_graph_from_edges(3, np.array([[1, 1]], np.uint32))
    with pytest.raises(ga.GAError):
        ga.build_graph_from_edges(4, np.array([[0, 1], [1, 0]], np.uint32))
    with pytest.raises(ga.GAError) as e:
        ga.load_graph("/nonexistent/graph.txt")
    assert e.value.name == "GA_ERR_IO"


def test_empty_and_tiny_graphs(ga, oracle, tmp_path):
    g = ga.build_graph_from_edges(0, np.zeros((0, 2), np.uint32))
    assert g.n == 0 and g.m == 0 and list(g.rowptr) == [0]
    g = ga.build_graph_from_edges(5, np.zeros((0, 2), np.uint32))
    assert g.m == 0 and list(g.rowptr) == [0] * 6
    p = tmp_path / "empty.txt"
    p.write_text("# nothing\n")
    g = ga.load_graph(str(p))
    o = oracle.load_graph(str(p))
    assert (g.n, g.m) == (o.n, o.m) == (1, 0)


def test_load_graph_parsing_rules(ga, oracle, tmp_path):
    p = tmp_path / "g.txt"
    p.write_text("# c\n% c\n\n1 2\n2\t1\n3 3\n4 7\nbad line\n7 4 extra\n  9 1\n0 5\n")
    g, o = ga.load_graph(str(p)), oracle.load_graph(str(p))
    assert (g.n, g.m) == (o.n, o.m) == (10, 4)
    assert np.array_equal(g.col, o.col) and np.array_equal(g.rowptr, o.rowptr)
    big = tmp_path / "big.txt"
    big.write_text("1 4294967296\n")
    with pytest.raises(ga.GAError) as e:
        ga.load_graph(str(big))
    assert e.value.name == "GA_ERR_INVALID_GRAPH"


def test_holme_kim_generator(ga):
    a = ga.gen_holme_kim(2000, 6, 7, 0.54, 0.3, seed=5)
    b = ga.gen_holme_kim(2000, 6, 7, 0.54, 0.3, seed=5)
    assert np.array_equal(a, b)                        # deterministic
    assert not np.array_equal(a, ga.gen_holme_kim(2000, 6, 7, 0.54, 0.3, seed=6))
    c = ga.canonical_edges(a)
    assert len(c) == len(a)                            # already unique, no self loops
    assert a.max() < 2000
    assert 6 * (2000 - 7) <= len(a) <= 7 * (2000 - 7)


def test_rmat_generator(ga):
    p = ga.gen_rmat(12, 40000, seed=3)
    assert p.shape == (40000, 2) and p.max() < 4096
    assert np.array_equal(p, ga.gen_rmat(12, 40000, seed=3))
    c = ga.canonical_edges(p)
    assert 0 < len(c) < 40000
    deg = np.bincount(c.reshape(-1), minlength=4096)
    assert deg.max() > 20 * max(1, np.median(deg[deg > 0]))   # skewed


def test_peel_helpers_match_oracle(ga, oracle):
    cases = [(100, 10**6, 1, 10), (0, 0, 0, 1), (4_000_000, 10**8, 1, 10), (10, 2**32, 1, 10), (10, 5, 1, 0),
             (10, 5, 2**20 + 1, 10), (2**31, 2**31, 1, 2**20)]
    for c in cases:
        assert ga.peel_arith_ok(*c)[0] == oracle.peel_arith_ok(*c)
    for c in [(5, 10, 0, 0), (5, 10, 1, 2), (1, 2, 1, 2), (3, 4, 1, 2)]:
        assert ga.peel_improves(*c) == oracle.peel_improves(*c)
    assert ga.density_value(3, 0) == 0.0 and ga.density_value(1197, 49) == 1197 / 49


def test_device_calls_fail_cleanly_without_gpu(ga):
    if ga.device_count() > 0:
        pytest.skip("a GPU is present")
    g = ga.build_graph_from_edges(3, np.array([[0, 1], [1, 2], [0, 2]], np.uint32))
    with pytest.raises(ga.GAError) as e:
        ga.DeviceGraph(g)
    assert e.value.name == "GA_ERR_NO_DEVICE"


def test_holme_kim_batch_generator(ga, oracle):
    b = ga.gen_holme_kim_batch(24, 64, 3000, 4.0, 16.0, 0.1, 0.7, seed=7)
    b2 = ga.gen_holme_kim_batch(24, 64, 3000, 4.0, 16.0, 0.1, 0.7, seed=7)
    assert np.array_equal(b.col, b2.col) and np.array_equal(b.rowptr, b2.rowptr)   # deterministic
    assert b.num_graphs == 24 and b.vtx_off[0] == 0 and b.edge_off[-1] == len(b.col)
    ns = np.diff(b.vtx_off)
    assert ns.min() >= 64 and ns.max() <= 3000
    for i in range(b.num_graphs):
        g = b.graph(i)
        # every packed graph is exactly the reference's orientation of its own edge set
        pairs = np.stack([g.src, g.col], 1)
        o = oracle.build_graph_from_edges(g.n, oracle.canonical_edges(pairs))
        assert np.array_equal(o.rowptr, g.rowptr) and np.array_equal(o.col, g.col)
        assert 1.5 <= 2 * g.m / g.n <= 17
    packed = ga.pack_batch([b.graph(i) for i in range(b.num_graphs)])
    assert np.array_equal(packed.rowptr, b.rowptr) and np.array_equal(packed.col, b.col)
