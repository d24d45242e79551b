"""GPU tests of the request loop (ga_server): every request served in a concurrent mix - folded into batch launches,
run on resident graphs, after evictions - returns exactly what the same request returns alone, and what the oracle
gives for that graph (triangle count, PeelResult fields (densest.h:46-59) with the whole removed_round array, kmax,
rounds and every core number of CoreLoopResult (dsg.h:687-691), the sets gpu_densest.cu:220-226 and
gpu_dsg.cu:283-289 read)."""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np
import pytest

from conftest import random_pairs

pytestmark = pytest.mark.gpu

EPS = [(1, 10), (1, 2)]


def _graphs(ga, seed):
    rng = np.random.default_rng(seed)
    gs = [ga.build_graph_from_edges(9, np.zeros((0, 2), np.uint32))]                        # no edges
    iu, iv = np.triu_indices(30, 1)
    gs.append(ga.build_graph_from_edges(30, np.stack([iu, iv], 1).astype(np.uint32)))     # a clique
    for _ in range(5):
        n = int(rng.integers(20, 300))
        gs.append(ga.build_graph_from_edges(n, ga.canonical_edges(random_pairs(rng, n, 0.1))))
    hk = ga.gen_holme_kim_batch(24, 64, 6000, 4.0, 20.0, 0.1, 0.7, seed=seed)               # small: folded
    gs += [hk.graph(i) for i in range(hk.num_graphs)]
    gs.append(ga.graph_from_pairs(40000, ga.gen_holme_kim(40000, 8, 24, 0.1, 0.7, seed=seed)))  # above the fold size
    gs.append(ga.graph_from_pairs(1 << 14, ga.gen_rmat(14, 16 << 14, seed=seed)))
    return gs


def _alone(ga, g):
    """Each request kind on its own device graph, one at a time (with the vertex arrays)."""
    out = {}
    with ga.DeviceGraph(g) as d:
        T = d.tc_count()
        out["tc"] = T
        for num, den in EPS:
            r = d.batch_peel(num, den)
            out[("peel", num, den)] = (T, r.best_num, r.best_den, r.best_round, r.rounds)
            out[("peel_array", num, den)] = r.removed_round
    with ga.DeviceGraph(g) as d:
        c = d.core_decomposition()
        out["core"] = (T, c.kmax, c.rounds)
        out["core_array"] = c.core
        out["bytes"] = d.device_bytes()   # resident with loop state and incidence lists
    return out


def _array_ok(ga, kind, num, den, r, a) -> bool:
    """The served vertex array equals the one of the request run alone."""
    if kind == ga.REQ_PEEL:
        return np.array_equal(r.peel.removed_round, a[("peel_array", num, den)])
    if kind == ga.REQ_CORE:
        return np.array_equal(r.core_numbers, a["core_array"])
    return True


def _key(kind, num, den):
    return "tc" if kind == 0 else ("peel", num, den) if kind == 1 else "core"


def _value(ga, kind, r):
    if kind == ga.REQ_TC:
        return r.triangles
    if kind == ga.REQ_PEEL:
        return (r.triangles, r.peel.best_num, r.peel.best_den, r.peel.best_round, r.peel.rounds)
    return (r.triangles, r.core[0], r.core[1])


def _mix(rng, ngraphs, requery):
    """Request list: every graph once per kind and eps, plus re-queries of random graphs, shuffled."""
    reqs = [(i, 0, 1, 1) for i in range(ngraphs)]
    reqs += [(i, 1, num, den) for i in range(ngraphs) for num, den in EPS]
    reqs += [(i, 2, 1, 1) for i in range(ngraphs)]
    extra = [reqs[j] for j in rng.integers(0, len(reqs), int(requery * len(reqs)))]
    reqs += extra
    return [reqs[j] for j in rng.permutation(len(reqs))]


@pytest.fixture(scope="module")
def served(ga, cuda_ok):
    gs = _graphs(ga, 5)
    alone = [_alone(ga, g) for g in gs]
    return gs, alone


def test_alone_matches_oracle(ga, oracle, served):
    gs, alone = served
    for g, a in zip(gs, alone):
        if g.m > 200000:
            continue
        assert a["tc"] == oracle.triangles_serial(g)
        for num, den in EPS:
            o = oracle.batch_peel(g, num, den)
            assert a[("peel", num, den)][1:] == (o.best_num, o.best_den, o.best_round, o.rounds)
            assert np.array_equal(a[("peel_array", num, den)], o.removed_round)
        core, kmax, rounds = oracle.core_levels(g)
        assert a["core"][1:] == (kmax, rounds)
        assert np.array_equal(a["core_array"], core)


@pytest.mark.parametrize("slots,fold,small,pin", [(4, 64, 0, 0), (1, 64, 1, 1), (6, 1, 3, 0), (3, 5, 2, 1)])
def test_mix_equals_alone(ga, served, slots, fold, small, pin):
    """pin = 1 keeps every graph's host copy page-locked (the path large graphs take)."""
    gs, alone = served
    rng = np.random.default_rng(slots * 100 + fold)
    reqs = _mix(rng, len(gs), 0.3)
    with ga.Server(slots=slots, fold_max_graphs=fold, small_slots=small, pin_min_edges=pin) as s:
        ids = [s.add_graph(g) for g in gs]
        # every other request also asks for its vertex array (removed_round / core numbers)
        tickets = [s.submit(ids[i], kind, num, den, want_array=j % 2 == 0)
                   for j, (i, kind, num, den) in enumerate(reqs)]
        for j, (t, (i, kind, num, den)) in enumerate(zip(tickets, reqs)):
            r = s.wait(t)
            assert r.status == 0, (i, kind)
            assert _value(ga, kind, r) == alone[i][_key(kind, num, den)], (i, kind, num, den, r.folded)
            if j % 2 == 0:
                assert _array_ok(ga, kind, num, den, r, alone[i]), (i, kind, num, den, r.folded)
        st = s.stats()
    assert st["submitted"] == st["completed"] == len(reqs)
    if fold > 1:
        assert st["folded_launches"] > 0
    assert st["resident_graphs"] > 0


def _wait(s, ticket, what):
    """The result within 300 s, or a failure that says where the request was: still queued (not admitted) or
    running (on a worker) - with the admission's reservation."""
    r = s.wait_for(ticket, 300.0)
    if r is None:   # written past pytest's capture: closing the server waits for the request too
        sys.__stderr__.write(f"{what}: not done after 300 s, server stats {s.stats()}\n")
        sys.__stderr__.flush()
    assert r is not None, (what, "not done after 300 s", s.stats())
    return r


def test_requery_hits_resident_graph(ga, served):
    gs, alone = served
    big = len(gs) - 1
    with ga.Server(slots=2) as s:
        gid = s.add_graph(gs[big])
        first = _wait(s, s.submit(gid, ga.REQ_TC), "count")
        again = _wait(s, s.submit(gid, ga.REQ_PEEL, 1, 10), "peel")
        core = _wait(s, s.submit(gid, ga.REQ_CORE), "cores")
    assert not first.resident_hit and again.resident_hit and core.resident_hit
    assert first.triangles == alone[big]["tc"]
    assert _value(ga, ga.REQ_PEEL, again) == alone[big][("peel", 1, 10)]
    assert _value(ga, ga.REQ_CORE, core) == alone[big]["core"]


def test_small_budget_evicts_and_still_matches(ga, served):
    """Two registrations of the largest graph under a budget that holds one of them with its loop state: requests
    alternate, graphs are evicted and uploaded again, results stay the same."""
    gs, alone = served
    big = len(gs) - 1
    budget = int(alone[big]["bytes"] * 1.5)
    rng = np.random.default_rng(9)
    with ga.Server(slots=2, fold_max_graphs=1, hbm_budget_bytes=budget) as s:
        ids = [s.add_graph(gs[big]), s.add_graph(gs[big])]
        reqs = [(c, kind) for _ in range(3) for c in (0, 1) for kind in (0, 1, 2)]
        reqs = [reqs[j] for j in rng.permutation(len(reqs))]
        tickets = [s.submit(ids[c], kind, 1, 10, want_array=True) for c, kind in reqs]
        for t, (c, kind) in zip(tickets, reqs):
            r = s.wait(t)
            assert r.status == 0, (c, kind)
            assert _value(ga, kind, r) == alone[big][_key(kind, 1, 10)]
            assert _array_ok(ga, kind, 1, 10, r, alone[big])
        st = s.stats()
    assert st["peak_reserved_bytes"] <= budget
    assert st["evictions"] > 0


def test_refusals(ga, served):
    gs, _ = served
    with ga.Server(hbm_budget_bytes=1 << 16) as s:
        with pytest.raises(ga.GAError) as e:
            s.add_graph(gs[-1])                              # can never fit the budget
        assert e.value.name == "GA_ERR_BUDGET"
        gid = s.add_graph(gs[0])
        with pytest.raises(ga.GAError):
            s.submit(gid + 100, ga.REQ_TC)                   # unknown graph
        with pytest.raises(ga.GAError):
            s.submit(gid, ga.REQ_PEEL, 1, 0)                 # eps denominator 0
        with pytest.raises(ga.GAError):
            s.wait(12345)                                    # unknown ticket
        short = np.zeros(max(gs[0].n - 1, 0), np.uint32)
        t = C.c_uint64(0)
        rc = ga.lib().ga_server_submit_out(s._h, gid, ga.REQ_CORE, 1, 1, short.ctypes.data if short.size else None,
                                           short.size, C.byref(t))
        assert ga.STATUS[rc] == "GA_ERR_INVALID_ARGUMENT"    # vertex array shorter than n
        t = s.submit(gid, ga.REQ_TC)
        r = s.wait(t)
        assert r.status == 0 and r.triangles == 0
        with pytest.raises(ga.GAError):
            s.wait(t)                                        # a result is handed out once
        t = s.submit(gid, ga.REQ_TC)
        while s.poll(t) is None:
            pass
        with pytest.raises(ga.GAError):
            s.poll(t)
