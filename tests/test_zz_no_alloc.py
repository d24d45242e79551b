"""ga_tc_count_noalloc: the triangle count for callers that cannot allocate device memory (their HBM is owned by
another allocator, or cudaMalloc's implicit synchronisation is not acceptable on their path). It must give the same
count as the allocating entry point ga_tc_count, call after call, although every call reuses the same fixed scratch
array compiled into the library. Collected last (file name) so that a failure here comes after all other tests."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(ga):
    f = ga.lib().ga_tc_count_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p, C.POINTER(C.c_uint64)]
    f.restype = C.c_int
    return f


def _count_noalloc(ga, torch, g, stream=None):
    rp = torch.from_numpy(g.rowptr.view(np.int32)).cuda()
    col = torch.from_numpy((g.col if g.m else np.zeros(1, np.uint32)).view(np.int32)).cuda()
    torch.cuda.synchronize()
    out = C.c_uint64(0)
    st = stream.cuda_stream if stream is not None else None
    rc = _noalloc(ga)(rp.data_ptr(), col.data_ptr(), g.n, g.m, 0, st, C.byref(out))
    return rc, out.value


def test_noalloc_matches_allocating_count_twice(ga, cuda_ok):
    import torch
    graphs = [
        ga.graph_from_pairs(3000, ga.gen_holme_kim(3000, 6, 7, 0.54, 0.5, seed=1)),
        ga.graph_from_pairs(1 << 15, ga.gen_rmat(15, 9 << 15, seed=4)),
        ga.graph_from_pairs(500, ga.gen_holme_kim(500, 3, 3, 0.0, 0.3, seed=2)),   # smaller after larger
    ]
    s = torch.cuda.Stream()
    for g in graphs:
        with ga.DeviceGraph(g) as d:
            want = d.tc_count()
        for call in range(2):                                   # two calls in a row share the scratch
            rc, got = _count_noalloc(ga, torch, g, stream=s if call else None)
            assert rc == 0, ga.lib().ga_last_error().decode()
            assert got == want


def test_noalloc_refusals(ga, cuda_ok):
    import torch
    f = _noalloc(ga)
    out = C.c_uint64(0)
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    # beyond the stated maximum: refused before anything is read or launched
    rc = f(dummy.data_ptr(), dummy.data_ptr(), 10, (4194304 + 1), 0, None, C.byref(out))
    assert ga.STATUS[rc] == "GA_ERR_CAPACITY"
    # an endpoint >= n: flagged on the device, no row followed
    g = ga.build_graph_from_edges(4, np.array([[0, 1], [1, 2], [0, 2], [2, 3]], np.uint32))
    bad = ga.Graph(g.n, g.m, g.rowptr.copy(), g.col.copy(), g.src, g.max_out_degree)
    bad.col[0] = 77
    rc, _ = _count_noalloc(ga, torch, bad)
    assert ga.STATUS[rc] == "GA_ERR_INVALID_GRAPH"
    rc, got = _count_noalloc(ga, torch, g)                      # the next call is clean again
    assert rc == 0 and got == 1
