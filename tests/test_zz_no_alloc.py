"""ga_tc_count_noalloc: the triangle count for callers that cannot allocate device memory (their HBM is owned by
another allocator, or cudaMalloc's implicit synchronisation is not acceptable on their path). It must give the same
count as the allocating entry point ga_tc_count, call after call, although every call reuses the same fixed scratch
array compiled into the library; after a first call on the device it must allocate nothing, so it still counts when
another allocator holds nearly all of the free HBM. Collected last (file name) so that a failure here comes after all
other tests."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_EDGES = 4194304
MAX_VERTICES = 4194304


def _noalloc(ga):
    f = ga.lib().ga_tc_count_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p, C.POINTER(C.c_uint64)]
    f.restype = C.c_int
    return f


def _upload(torch, g):
    rp = torch.from_numpy(g.rowptr.view(np.int32)).cuda()
    col = torch.from_numpy((g.col if g.m else np.zeros(1, np.uint32)).view(np.int32)).cuda()
    torch.cuda.synchronize()
    return rp, col


def _call(ga, rp, col, n, m, stream=None):
    out = C.c_uint64(0)
    st = stream.cuda_stream if stream is not None else None
    rc = _noalloc(ga)(rp.data_ptr(), col.data_ptr(), n, m, 0, st, C.byref(out))
    return rc, out.value


def _count_noalloc(ga, torch, g, stream=None):
    rp, col = _upload(torch, g)
    return _call(ga, rp, col, g.n, g.m, stream)


def _warm_up(ga, torch):
    """The documented first call (n = m = 0): loads the library's code on the device and finds the array."""
    rp = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc, got = _call(ga, rp, rp, 0, 0)
    assert rc == 0 and got == 0, ga.lib().ga_last_error().decode()


def _csr(n, rows):
    """A CSR given row by row, in the order given (no orientation applied)."""
    rowptr = np.zeros(n + 1, np.uint32)
    for u, r in enumerate(rows):
        rowptr[u + 1] = rowptr[u] + len(r)
    col = np.array([x for r in rows for x in r], np.uint32)
    return rowptr, col


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
    # beyond the stated maxima: refused before anything is read or launched
    rc = f(dummy.data_ptr(), dummy.data_ptr(), 10, MAX_EDGES + 1, 0, None, C.byref(out))
    assert ga.STATUS[rc] == "GA_ERR_CAPACITY"
    rc = f(dummy.data_ptr(), dummy.data_ptr(), MAX_VERTICES + 1, 0, 0, None, C.byref(out))
    assert ga.STATUS[rc] == "GA_ERR_CAPACITY"
    # an endpoint >= n: flagged on the device, no row followed
    g = ga.build_graph_from_edges(4, np.array([[0, 1], [1, 2], [0, 2], [2, 3]], np.uint32))
    bad = ga.Graph(g.n, g.m, g.rowptr.copy(), g.col.copy(), g.src, g.max_out_degree)
    bad.col[0] = 77
    rc, _ = _count_noalloc(ga, torch, bad)
    assert ga.STATUS[rc] == "GA_ERR_INVALID_GRAPH"
    rc, got = _count_noalloc(ga, torch, g)                      # the next call is clean again
    assert rc == 0 and got == 1


def test_noalloc_refuses_other_orientations(ga, cuda_ok):
    """Sorted rows without self loops are not enough: a cyclic orientation (0->1->2->0) would count 0 triangles and a
    symmetric CSR 6 per triangle, so both are refused; the (degree, id) orientation of the same triangle counts 1."""
    import torch
    cases = {
        "cyclic": _csr(3, [[1], [2], [0]]),
        "symmetric": _csr(3, [[1, 2], [0, 2], [0, 1]]),
        "id order against degree order": _csr(4, [[1, 2, 3], [2], [], []]),   # 0 has degree 3, so 1->0 is required
    }
    for name, (rowptr, col) in cases.items():
        g = ga.Graph(len(rowptr) - 1, len(col), rowptr, col, np.zeros(len(col), np.uint32), 0)
        rc, _ = _count_noalloc(ga, torch, g)
        assert ga.STATUS[rc] == "GA_ERR_INVALID_GRAPH", name
        assert "orientation" in ga.lib().ga_last_error().decode(), name
    g = ga.build_graph_from_edges(3, np.array([[0, 1], [1, 2], [0, 2]], np.uint32))
    rc, got = _count_noalloc(ga, torch, g)
    assert rc == 0 and got == 1


def test_noalloc_allocates_nothing_after_first_call(ga, cuda_ok):
    """After the documented first call, a call leaves the device's free memory unchanged, and it still counts when
    another allocator (torch here) holds all of the free HBM but a small margin."""
    import torch
    _warm_up(ga, torch)
    g = ga.graph_from_pairs(1 << 16, ga.gen_rmat(16, 9 << 16, seed=7))
    with ga.DeviceGraph(g) as d:
        want = d.tc_count()
    rp, col = _upload(torch, g)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        rc, got = _call(ga, rp, col, g.n, g.m, stream)
        assert rc == 0 and got == want, ga.lib().ga_last_error().decode()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    # another allocator claims the free HBM in chunks, leaving between 256 and 320 MiB
    margin, hog = 256 << 20, []
    try:
        for chunk in (1 << 30, 64 << 20):
            while torch.cuda.mem_get_info()[0] > margin + chunk:
                hog.append(torch.empty(chunk, dtype=torch.uint8, device="cuda"))
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] <= margin + (64 << 20)
        for _ in range(2):
            rc, got = _call(ga, rp, col, g.n, g.m, stream)
            assert rc == 0 and got == want, ga.lib().ga_last_error().decode()
    finally:
        hog.clear()
        torch.cuda.empty_cache()
