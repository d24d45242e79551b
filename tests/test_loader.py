"""Loaders: the parallel text path of ga_load_graph against the reference's own load_graph (graph.h:71-96, compiled
here) and the oracle on inputs that exercise every line rule, including the cases that route to the sequential
fgets path (a line longer than fgets' 511 bytes, a NUL byte); and the binary CSR files (round trip, damage and
foreign files refused)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import FIXTURES, fixture_path

TRICKY = (
    "# comment\n% comment\n\n"
    "1 2\n2\t1\n3 3\n4 7\n  9 1\n\t5\t6\t\n+8 +2\n-0 3\n"
    "bad line\n7 4 extra\n 1x 2\n10 11\r\n\r\n12    13\n"
    " # not a comment for the first-byte rule, but no number either\n"
    "%10 20\n#1 2\n14 15"                       # last line without a newline
)


def _same(g, o):
    assert (g.n, g.m, g.max_out_degree) == (o.n, o.m, o.max_out_degree)
    assert np.array_equal(g.rowptr, o.rowptr) and np.array_equal(g.col, o.col) and np.array_equal(g.src, o.src)


def _write(tmp_path, name, data: bytes):
    p = tmp_path / name
    p.write_bytes(data)
    return str(p)


def test_line_rules_match_reference(ga, oracle, reference, tmp_path):
    p = _write(tmp_path, "tricky.txt", TRICKY.encode())
    g = ga.load_graph(p)
    _same(g, reference.load_graph(p))
    _same(g, oracle.load_graph(p))


def test_long_line_and_nul_take_the_fgets_path(ga, reference, tmp_path):
    # a 600-byte line is read by fgets as two chunks: "1 2 <spaces>" and "<spaces>3 4\n" -> two pairs
    long_line = b"1 2" + b" " * 600 + b"3 4\n"
    p = _write(tmp_path, "long.txt", b"5 6\n" + long_line + b"7 8\n")
    g = ga.load_graph(p)
    _same(g, reference.load_graph(p))
    assert g.m == 4
    p = _write(tmp_path, "nul.txt", b"1 2\n3\x00 4\n5 6\n")
    _same(ga.load_graph(p), reference.load_graph(p))


def test_large_file_parallel_chunks(ga, reference, tmp_path):
    """Several MB, so the file is cut into one range per host thread at line starts."""
    rng = np.random.default_rng(3)
    n = 200_000
    e = rng.integers(0, n, (400_000, 2))
    lines = [f"{a}\t{b}" if i % 7 else f"  {a} {b} x" for i, (a, b) in enumerate(e)]
    lines.insert(1000, "# mid-file comment")
    p = _write(tmp_path, "big.txt", ("\n".join(lines) + "\n").encode())
    g = ga.load_graph(p)
    _same(g, reference.load_graph(p))


@pytest.mark.parametrize("text", ["-1 5\n", "1 4294967296\n", "99999999999999999999999 3\n"])
def test_ids_beyond_uint32_are_refused(ga, text, tmp_path):
    p = _write(tmp_path, "big.txt", ("1 2\n" + text).encode())
    with pytest.raises(ga.GAError) as e:
        ga.load_graph(p)
    assert e.value.name == "GA_ERR_INVALID_GRAPH"


def test_equal_out_of_range_pair_is_skipped(ga, reference, tmp_path):
    # a == b is tested before the range: "-1 -1" is a self loop and is dropped like in graph.h:84
    p = _write(tmp_path, "g.txt", b"-1 -1\n1 2\n")
    _same(ga.load_graph(p), reference.load_graph(p))


@pytest.mark.parametrize("name", FIXTURES)
def test_binary_round_trip(ga, tmp_path, name):
    g = ga.load_graph(fixture_path(name))
    p = str(tmp_path / (name + ".gacsr"))
    ga.save_csr(g, p)
    _same(ga.load_csr(p), g)


def test_binary_round_trip_edge_cases(ga, tmp_path):
    for n, pairs in ((0, []), (1, []), (7, []), (3, [[0, 1], [1, 2], [0, 2]])):
        g = ga.build_graph_from_edges(n, np.array(pairs, np.uint32).reshape(-1, 2))
        p = str(tmp_path / f"g{n}.gacsr")
        ga.save_csr(g, p)
        _same(ga.load_csr(p), g)


def test_binary_damage_is_refused(ga, tmp_path):
    g = ga.load_graph(fixture_path("t_pl400"))
    p = tmp_path / "g.gacsr"
    ga.save_csr(g, str(p))
    raw = bytearray(p.read_bytes())
    flipped = bytearray(raw)
    flipped[-5] ^= 0x01                                   # one bit of col
    cases = {"flip.gacsr": bytes(flipped), "trunc.gacsr": bytes(raw[:-4]), "magic.gacsr": b"GACSR002" + bytes(raw[8:]),
             "text.gacsr": b"1 2\n"}
    for fname, data in cases.items():
        q = _write(tmp_path, fname, data)
        with pytest.raises(ga.GAError) as e:
            ga.load_csr(q)
        assert e.value.name == "GA_ERR_INVALID_GRAPH", fname
    with pytest.raises(ga.GAError) as e:
        ga.load_csr(str(tmp_path / "missing.gacsr"))
    assert e.value.name == "GA_ERR_IO"


def test_save_refuses_invalid_csr(ga, tmp_path):
    g = ga.load_graph(fixture_path("t_er300"))
    bad = ga.Graph(g.n, g.m, g.rowptr.copy(), g.col[::-1].copy(), g.src, g.max_out_degree)   # rows unsorted
    with pytest.raises(ga.GAError) as e:
        ga.save_csr(bad, str(tmp_path / "bad.gacsr"))
    assert e.value.name == "GA_ERR_INVALID_GRAPH"
    # a valid CSR shape whose edges point from higher to lower (degree, id): orientation refused
    tri = ga.Graph(3, 1, np.array([0, 0, 1, 1], np.uint32), np.array([0], np.uint32), np.array([1], np.uint32), 1)
    with pytest.raises(ga.GAError):
        ga.save_csr(tri, str(tmp_path / "bad2.gacsr"))
