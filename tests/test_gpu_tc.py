"""GPU parity: triangle count, per-edge and per-vertex support, alive-subgraph participation (through the C ABI)
against the oracle and the reference's golden outputs. Integer work: bit-exact equality everywhere."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import FIXTURES, fixture_path, golden_arrays, hub_pairs, random_pairs

pytestmark = pytest.mark.gpu

# kernel configurations that force every path: default (light + heavy bins), plain merge kernel, tiny light bin with
# a small heavy table (heavy anchors and the global binary-search fallback; option 8 keeps counts on hash sets),
# small work items (many items/anchor)
CONFIGS = {
    "auto": {},
    "plain": {1: 1},
    "heavy_global": {6: 8, 5: 3, 8: 1},
    "heavy_table": {6: 4, 5: 10, 8: 1},
    # counts of heavy anchors against bitmaps of up to 1,024 places; wider anchors binary-search the global row
    "heavy_bitmap": {6: 4, 5: 3},
    "small_items": {4: 16},
    # light bin up to out-degree 256: in the support modes anchors above 128 fall back to binary search
    "light_256": {6: 256, 1: 2},
}


def _dev(ga, g, cfg):
    d = ga.DeviceGraph(g)
    for opt, val in CONFIGS[cfg].items():
        d.set_option(opt, val)
    return d


def _check_all(ga, oracle, g, cfg, rng):
    T = oracle.triangles_serial(g)
    _, sup = oracle.edge_support(g)
    _, deg = oracle.triangle_degrees(g)
    with _dev(ga, g, cfg) as d:
        assert d.tc_count() == T
        assert d.tc_count() == T                                  # repeat launches are identical
        Ts, gsup = d.support_edges()
        assert Ts == T and np.array_equal(gsup, sup)
        Tv, gdeg = d.support_vertices()
        assert Tv == T and np.array_equal(gdeg, deg)
        for pa in (1.0, 0.9, 0.6, 0.3, 0.05, 0.0):                 # emu_densest.cpp:97-114 masks
            alive = (rng.random(g.n) < pa).astype(np.uint8)
            Ta, tri = d.participation(alive)
            To, trio = oracle.participation(g, alive)
            assert Ta == To and np.array_equal(tri, trio)


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("cfg", list(CONFIGS))
def test_fixtures(ga, oracle, golden, cuda_ok, name, cfg):
    g = ga.load_graph(fixture_path(name))
    arr = golden_arrays(name)
    with _dev(ga, g, cfg) as d:
        assert d.tc_count() == golden[name]["brute_force_triangles"]
        assert np.array_equal(d.support_edges()[1], arr["sup"])
        assert np.array_equal(d.support_vertices()[1], arr["deg"])
    _check_all(ga, oracle, g, cfg, np.random.default_rng(7))


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("cfg", list(CONFIGS))
def test_random_graphs(ga, oracle, cuda_ok, seed, cfg):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(50, 700))
    g = ga.build_graph_from_edges(n, ga.canonical_edges(random_pairs(rng, n, float(rng.choice([0.02, 0.1, 0.3])))))
    _check_all(ga, oracle, g, cfg, rng)


@pytest.mark.parametrize("cfg", ["auto", "heavy_global", "plain"])
def test_hub_graphs(ga, oracle, cuda_ok, cfg):
    rng = np.random.default_rng(11)
    for _ in range(4):
        n, raw = hub_pairs(rng, int(rng.integers(1, 4)), int(rng.integers(40, 400)), int(rng.integers(8, 40)))
        g = ga.build_graph_from_edges(n, ga.canonical_edges(raw))
        _check_all(ga, oracle, g, cfg, rng)


def _hash_class(ids: np.ndarray, bits: int) -> np.ndarray:
    """The table bucket of each id at 2^bits buckets (the multiplicative hash of the count kernel's tables)."""
    return ((ids.astype(np.uint64) * 2654435761) & 0xFFFFFFFF) >> (32 - bits)


def _colliding_graph(rng: np.random.Generator, bucket: int) -> tuple[int, np.ndarray]:
    """An anchor v whose 100 out-neighbours X all hash to one bucket of its table (256 two-slot buckets for 100 keys,
    so they fill a chain of 50 buckets, wrapping past the last bucket when `bucket` is 255), and 40 in-neighbours
    whose probe lists mix members of X (hits at every chain position) with 60 ids Y of the same bucket that are not
    in the table (misses that must walk the whole chain). Fillers give X and Y the higher degree, so v -> x and the
    lists of u -> v reach them."""
    n = 1 << 16
    ids = np.arange(n, dtype=np.int64)
    cls = ids[_hash_class(ids, 8) == bucket]
    rng.shuffle(cls)
    X, Y = cls[:100], cls[100:160]
    rest = np.setdiff1d(ids, cls)
    v, U, F = rest[0], rest[1:41], rest[41:241]
    pairs = [(v, x) for x in X]
    for u in U:
        pairs.append((u, v))
        pairs += [(u, x) for x in rng.choice(X, 30, replace=False)]
        pairs += [(u, y) for y in rng.choice(Y, 30, replace=False)]
    pairs += [(f, z) for f in F for z in np.concatenate([X, Y])]
    return n, np.array(pairs, dtype=np.uint32)


@pytest.mark.parametrize("cfg", list(CONFIGS))
def test_colliding_keys(ga, oracle, cuda_ok, cfg):
    """Table keys that all land in one bucket: the search must follow the chain of full buckets a key moved along
    when the table was built (hits anywhere in it, misses to its end), also where it wraps past the last bucket."""
    rng = np.random.default_rng(5)
    for bucket in (5, 255):
        n, raw = _colliding_graph(rng, bucket)
        g = ga.build_graph_from_edges(n, ga.canonical_edges(raw))
        assert oracle.triangles_serial(g) == 40 * 30
        _check_all(ga, oracle, g, cfg, rng)


@pytest.mark.parametrize("cfg", list(CONFIGS))
def test_clique_uses_heavy_bin(ga, oracle, cuda_ok, cfg):
    n = 640                                                       # out-degrees up to 639 > 256: heavy anchors
    iu, iv = np.triu_indices(n, 1)
    g = ga.build_graph_from_edges(n, np.stack([iu, iv], 1).astype(np.uint32))
    with _dev(ga, g, cfg) as d:
        assert d.tc_count() == n * (n - 1) * (n - 2) // 6
        T, deg = d.support_vertices()
        assert np.all(deg == (n - 1) * (n - 2) // 2)
        T, sup = d.support_edges()
        assert np.all(sup == n - 2)


def test_holme_kim_c1_shape(ga, oracle, cuda_ok):
    """The 8,298-vertex Holme-Kim graph (12 edges per new vertex, p = 0.5), ids permuted from the seed."""
    g = ga.graph_from_pairs(8298, ga.gen_holme_kim(8298, 12, 12, 0.0, 0.5, seed=1))
    _check_all(ga, oracle, g, "auto", np.random.default_rng(3))
    _check_all(ga, oracle, g, "plain", np.random.default_rng(3))


def test_rmat_skewed(ga, oracle, cuda_ok):
    g = ga.graph_from_pairs(1 << 14, ga.gen_rmat(14, 9 * (1 << 14), seed=2))
    _check_all(ga, oracle, g, "auto", np.random.default_rng(4))


def test_edge_cases(ga, oracle, cuda_ok):
    cases = [
        (0, np.zeros((0, 2), np.uint32)),
        (1, np.zeros((0, 2), np.uint32)),
        (7, np.zeros((0, 2), np.uint32)),
        (3, np.array([[0, 1], [1, 2], [0, 2]], np.uint32)),
        (5, np.array([[0, 1], [1, 2], [2, 3], [3, 4]], np.uint32)),          # a path: no triangle
        (300, np.array([[0, i] for i in range(1, 300)], np.uint32)),        # a star: no triangle
    ]
    for n, p in cases:
        g = ga.build_graph_from_edges(n, p)
        with ga.DeviceGraph(g) as d:
            assert d.tc_count() == oracle.triangles_serial(g)
            assert np.array_equal(d.support_edges()[1], oracle.edge_support(g)[1])
            assert np.array_equal(d.support_vertices()[1], oracle.triangle_degrees(g)[1])


def test_invalid_csr_rejected(ga, cuda_ok):
    good = ga.build_graph_from_edges(4, np.array([[0, 1], [1, 2], [0, 2], [2, 3]], np.uint32))
    bad = ga.Graph(good.n, good.m, good.rowptr.copy(), good.col.copy(), good.src, good.max_out_degree)
    bad.col[0] = 9                                                   # endpoint >= n
    with pytest.raises(ga.GAError) as e:
        ga.DeviceGraph(bad)
    assert e.value.name == "GA_ERR_INVALID_GRAPH"
    # both directions of an undirected edge: valid rows, but not a (degree, id) orientation
    rp = np.array([0, 1, 2], np.uint32)
    col = np.array([1, 0], np.uint32)
    d = ga.DeviceGraph(ga.Graph(2, 2, rp, col, np.array([0, 1], np.uint32), 1))
    with pytest.raises(ga.GAError) as e:
        d.tc_count()
    assert e.value.name == "GA_ERR_INVALID_GRAPH"
    d.close()


def test_device_create_and_streams(ga, oracle, cuda_ok):
    import torch
    g = ga.graph_from_pairs(2000, ga.gen_holme_kim(2000, 5, 5, 0.0, 0.5, seed=9))
    rp = torch.from_numpy(g.rowptr.astype(np.int32)).cuda()
    col = torch.from_numpy(g.col.astype(np.int32)).cuda()
    s = torch.cuda.Stream()
    with ga.DeviceGraph.from_device(rp.data_ptr(), col.data_ptr(), g.n, g.m, 0, s.cuda_stream) as d:
        assert d.tc_count() == oracle.triangles_serial(g)
        d.set_stream(None)
        assert d.tc_count() == oracle.triangles_serial(g)
        sup = torch.zeros(g.m, dtype=torch.int32, device="cuda")
        assert d.support_edges_device(sup.data_ptr()) == oracle.triangles_serial(g)
        assert np.array_equal(sup.cpu().numpy().view(np.uint32), oracle.edge_support(g)[1])
        assert d.device_bytes() > 0


@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_shards_partition_the_triangles(ga, oracle, cuda_ok, kernel):
    """One shard per GPU in a multi-GPU count: the shards' partial counts sum to the whole count for any number of
    shards, with either kernel (0 = automatic: the hash kernel for shards)."""
    rng = np.random.default_rng(17)
    graphs = [ga.load_graph(fixture_path("t_pl900")),
              ga.graph_from_pairs(1 << 13, ga.gen_rmat(13, 16 << 13, seed=3)),
              ga.build_graph_from_edges(200, ga.canonical_edges(random_pairs(rng, 200, 0.3)))]
    import torch
    for g in graphs:
        T = oracle.triangles_serial(g)
        with ga.DeviceGraph(g) as d:
            if kernel:
                d.set_option(ga.OPT_TC_KERNEL, kernel)
            for k in (1, 2, 3, 8, 64):
                parts = [d.tc_count_shard(s, k) for s in range(k)]
                assert sum(parts) == T, (k, parts)
            out = torch.zeros(4, dtype=torch.int64, device="cuda")
            for s in range(4):
                d.tc_count_shard_async(s, 4, out[s:].data_ptr())
            torch.cuda.synchronize()
            assert int(out.sum()) == T
            with pytest.raises(ga.GAError):
                d.tc_count_shard(3, 3)


def test_one_handle_from_many_threads(ga, oracle, cuda_ok):
    """Calls on one ga_graph from several host threads are serialised by the handle's lock: every call returns the
    same results as a lone call (the counts, supports and peeling share the handle's scratch and stream)."""
    import threading
    g = ga.graph_from_pairs(1 << 12, ga.gen_rmat(12, 16 << 12, seed=4))
    T = oracle.triangles_serial(g)
    _, sup = oracle.edge_support(g)
    o = oracle.batch_peel(g, 1, 10)
    errors = []
    with ga.DeviceGraph(g) as d:
        def work(i):
            try:
                for _ in range(5):
                    if i % 3 == 0:
                        assert d.tc_count() == T
                    elif i % 3 == 1:
                        t, s = d.support_edges()
                        assert t == T and np.array_equal(s, sup)
                    else:
                        r = d.batch_peel(1, 10)
                        assert (r.best_num, r.best_den, r.rounds) == (o.best_num, o.best_den, o.rounds)
            except Exception as e:   # reported below: an assert in a thread does not fail the test by itself
                errors.append(repr(e))
        threads = [threading.Thread(target=work, args=(i,)) for i in range(6)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    assert not errors, errors


def test_autotuner_choices(ga, oracle, cuda_ok):
    """The autotuner picks a kernel, bin cutoff and item work per degree-distribution signature; every candidate it
    times gives the oracle's count, options set by the caller are kept, and a second graph with the same signature
    takes the cached choice without timing."""
    graphs = [ga.graph_from_pairs(1 << 15, ga.gen_rmat(15, 9 << 15, seed=21)),
              ga.graph_from_pairs(50000, ga.gen_holme_kim(50000, 6, 7, 0.54, 0.3, seed=22))]
    for g in graphs:
        want = oracle.triangles_omp(g)
        with ga.DeviceGraph(g) as d:
            assert d.tc_count() == want
            t = d.tuning()
            assert t["kernel"] in ("plain", "hash") and t["light_max_deg"] in (32, 64, 128, 256)
            assert t["item_work"] in (1024, 4096, 16384) and t["measured_ms"] >= 0   # 0: an earlier graph's choice
            _, sup = d.support_edges()
            assert np.array_equal(sup, oracle.edge_support(g)[1])
        with ga.DeviceGraph(g) as d:                 # same signature: from the cache
            assert d.tc_count() == want
            t2 = d.tuning()
            assert t2["measured_ms"] == 0 and t2["signature"] == t["signature"]
            assert (t2["kernel"], t2["light_max_deg"], t2["item_work"]) == (t["kernel"], t["light_max_deg"],
                                                                             t["item_work"])
        with ga.DeviceGraph(g) as d:                 # caller's options stay
            d.set_option(ga.OPT_LIGHT_MAX_DEG, 64)
            d.set_option(ga.OPT_ITEM_WORK, 2048)
            assert d.tc_count() == want
            t3 = d.tuning()
            assert (t3["light_max_deg"], t3["item_work"]) == (64, 2048)
