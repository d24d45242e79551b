"""graph_analyzer_b200 - the triangle path of graph_analyzer on one B200 (sm_100a), Python host layer.

A thin ctypes layer over ``libga_b200.so`` (the C ABI declared in include/graph_analyzer_b200.h). Names follow the
reference's C++ surface (VijayPraneethSai/graph_analyzer, paths relative to that project):

=====================================  ==========================================================================
reference                              here
=====================================  ==========================================================================
``struct Graph`` (graph.h:19-26)        :class:`Graph`
``build_graph_from_edges`` (graph.h:38) :func:`build_graph_from_edges`
``load_graph`` (graph.h:71)             :func:`load_graph`
``PeelResult`` (densest.h:46-59)        :class:`PeelResult` (``==`` compares like ``operator==``)
``density_value`` / ``peel_arith_ok``   :func:`density_value`, :func:`peel_arith_ok`, :func:`peel_improves`
 / ``peel_improves`` (densest.h:62-78)
count kernels driven by gpu_tc.cu       :meth:`DeviceGraph.tc_count` / :func:`gpu_triangles`
``tc_per_vertex_alive`` (kernels.cuh)   :meth:`DeviceGraph.participation`
``triangle_degrees`` (dsg.h:82)         :meth:`DeviceGraph.support_vertices`
``for_each_triangle`` (dsg.h:67)        :meth:`DeviceGraph.support_edges` (per-edge support)
``batch_peel_loop`` (densest.h:279)     :meth:`DeviceGraph.batch_peel` / :func:`gpu_batch_peel`
``core_decomp_loop_inc`` (dsg.h:724)    :meth:`DeviceGraph.core_decomposition` / :func:`gpu_core_decomposition`
=====================================  ==========================================================================

There is no CPU fallback: every count comes from the CUDA library, and a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "GAError", "Graph", "PeelResult", "CoreResult", "DeviceGraph", "build_graph_from_edges", "load_graph",
    "canonical_edges", "gen_holme_kim", "gen_rmat", "permute_ids", "density_value", "peel_arith_ok",
    "peel_improves", "gpu_triangles", "gpu_batch_peel", "gpu_core_decomposition", "lib", "device_count",
    "OPT_TC_KERNEL", "OPT_LOOP_MODE", "OPT_MAX_ROUNDS", "OPT_ITEM_WORK", "OPT_HEAVY_TABLE_BITS",
    "OPT_LIGHT_MAX_DEG", "OPT_UPDATE_MODE", "OPT_COUNT_BITMAP", "HostBatch", "DeviceBatch", "BatchPeel", "pack_batch",
    "gen_holme_kim_batch",
]

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "libga_b200.so")

OPT_TC_KERNEL, OPT_LOOP_MODE, OPT_MAX_ROUNDS, OPT_ITEM_WORK, OPT_HEAVY_TABLE_BITS, OPT_LIGHT_MAX_DEG = 1, 2, 3, 4, 5, 6
OPT_UPDATE_MODE = 7
OPT_COUNT_BITMAP = 8

STATUS = {
    0: "GA_OK", 1: "GA_ERR_INVALID_ARGUMENT", 2: "GA_ERR_INVALID_GRAPH", 3: "GA_ERR_CUDA",
    4: "GA_ERR_OUT_OF_MEMORY", 5: "GA_ERR_ARITH", 6: "GA_ERR_ROUND_LIMIT", 7: "GA_ERR_IO", 8: "GA_ERR_NO_DEVICE",
    9: "GA_ERR_DEVICE_CHECK", 10: "GA_ERR_BUDGET", 11: "GA_ERR_CAPACITY", 12: "GA_ERR_NOT_READY",
}


class GAError(RuntimeError):
    """A ga_status other than GA_OK; ``.status`` is the code, ``.name`` its symbol."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.name = STATUS.get(status, f"status {status}")
        super().__init__(f"{self.name}: {message}")


_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_vp = C.c_void_p


class _HostGraph(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint32), ("max_out_degree", C.c_uint32),
                ("rowptr", C.POINTER(C.c_uint32)), ("col", C.POINTER(C.c_uint32)), ("src", C.POINTER(C.c_uint32))]


class _PeelRes(C.Structure):
    _fields_ = [("best_num", C.c_uint64), ("best_den", C.c_uint64), ("best_round", C.c_uint32),
                ("rounds", C.c_uint32)]


class _CoreRes(C.Structure):
    _fields_ = [("kmax", C.c_uint32), ("rounds", C.c_uint32)]


class _DsgRes(C.Structure):
    _fields_ = [("tri", C.c_uint64), ("verts", C.c_uint64), ("flow_calls", C.c_uint32),
                ("components_searched", C.c_uint32), ("shrinks", C.c_uint32), ("reserved", C.c_uint32)]


class _DsgSeed(C.Structure):
    _fields_ = [("set", _vp), ("set_len", C.c_uint64), ("tri", C.c_uint64), ("verts", C.c_uint64)]


class _ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_uint64), ("slots", C.c_uint32),
                ("fold_max_graphs", C.c_uint32), ("fold_max_edges", C.c_uint32), ("small_slots", C.c_uint32),
                ("pin_min_edges", C.c_uint32)]


class _RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("triangles", C.c_uint64), ("peel", _PeelRes), ("core", _CoreRes),
                ("queue_ms", C.c_double), ("run_ms", C.c_double), ("folded", C.c_uint32),
                ("resident_hit", C.c_uint32)]


class _ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "folded_launches", "evictions",
                                          "resident_graphs", "resident_bytes", "peak_reserved_bytes", "queued",
                                          "running", "reserved_bytes")]


class _HostBatch(C.Structure):
    _fields_ = [("num_graphs", C.c_uint32), ("total_vertices", C.c_uint64), ("total_edges", C.c_uint64),
                ("vtx_off", C.POINTER(C.c_uint64)), ("edge_off", C.POINTER(C.c_uint64)),
                ("rowptr", C.POINTER(C.c_uint32)), ("col", C.POINTER(C.c_uint32))]


# (name, argtypes) of every exported entry point; the library must export all of them.
class _Tuning(C.Structure):
    _fields_ = [("kernel", C.c_uint32), ("light_max_deg", C.c_uint32), ("item_work", C.c_uint32),
                ("reserved", C.c_uint32), ("signature", C.c_uint64), ("measured_ms", C.c_double),
                ("heavy_items", C.c_uint64), ("light_items", C.c_uint64)]


def _tuning_dict(t: _Tuning) -> dict:
    return {"kernel": {1: "plain", 2: "hash"}.get(t.kernel, str(t.kernel)), "light_max_deg": t.light_max_deg,
            "item_work": t.item_work, "signature": f"{t.signature:016x}", "measured_ms": t.measured_ms,
            "heavy_items": t.heavy_items, "light_items": t.light_items}


SIGNATURES: dict[str, list] = {
    "ga_status_string": [C.c_int],
    "ga_last_error": [],
    "ga_device_count": [C.POINTER(C.c_int)],
    "ga_host_pinned_alloc": [C.c_uint64, C.POINTER(_vp)],
    "ga_host_pinned_free": [_vp],
    "ga_canonical_edges": [_u32p, C.c_uint64, C.POINTER(C.c_uint64)],
    "ga_build_graph_from_edges": [C.c_uint32, _u32p, C.c_uint32, _u32p, _u32p, _u32p, C.POINTER(C.c_uint32)],
    "ga_host_graph_from_edges": [C.c_uint32, _u32p, C.c_uint64, C.c_int, C.POINTER(C.POINTER(_HostGraph))],
    "ga_load_graph": [C.c_char_p, C.POINTER(C.POINTER(_HostGraph))],
    "ga_save_csr": [C.c_char_p, C.c_uint32, C.c_uint32, _u32p, _vp],
    "ga_load_csr": [C.c_char_p, C.POINTER(C.POINTER(_HostGraph))],
    "ga_host_graph_free": [C.POINTER(_HostGraph)],
    "ga_gen_holme_kim": [C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint64, _u32p, C.c_uint64,
                         C.POINTER(C.c_uint64)],
    "ga_gen_rmat": [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64, _u32p],
    "ga_permute_ids": [_u32p, C.c_uint64, C.c_uint32, C.c_uint64],
    "ga_graph_create": [_vp, _vp, C.c_uint32, C.c_uint32, C.c_int, _vp, C.POINTER(_vp)],
    "ga_graph_create_device": [_vp, _vp, C.c_uint32, C.c_uint32, C.c_int, _vp, C.POINTER(_vp)],
    "ga_graph_destroy": [_vp],
    "ga_graph_set_stream": [_vp, _vp],
    "ga_graph_device_bytes": [_vp, C.POINTER(C.c_uint64)],
    "ga_graph_prepare": [_vp],
    "ga_graph_set_option": [_vp, C.c_int, C.c_int64],
    "ga_tc_count": [_vp, C.POINTER(C.c_uint64)],
    "ga_tc_count_async": [_vp, _vp],
    "ga_tc_count_shard": [_vp, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64)],
    "ga_tc_count_shard_async": [_vp, C.c_uint32, C.c_uint32, _vp],
    "ga_tc_support_edges": [_vp, _vp, C.POINTER(C.c_uint64)],
    "ga_tc_support_edges_device": [_vp, _vp, C.POINTER(C.c_uint64)],
    "ga_tc_support_vertices": [_vp, _vp, C.POINTER(C.c_uint64)],
    "ga_tc_participation": [_vp, _vp, _vp, C.POINTER(C.c_uint64)],
    "ga_core_level_density": [_vp, _vp, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
    "ga_graph_tuning": [_vp, C.POINTER(_Tuning)],
    "ga_batch_tuning": [_vp, C.POINTER(_Tuning)],
    "ga_batch_peel": [_vp, C.c_uint64, C.c_uint64, C.POINTER(_PeelRes), _vp],
    "ga_core_decomposition": [_vp, _vp, C.POINTER(_CoreRes)],
    "ga_greedy_pp": [_vp, C.c_uint32, C.POINTER(_DsgRes), _vp, _vp],
    "ga_core_exact": [_vp, _vp, C.c_int, C.POINTER(_DsgSeed), C.POINTER(_DsgRes), _vp],
    "ga_exact_densest": [_vp, C.POINTER(_DsgRes), _vp],
    "ga_greedy_pp_host": [C.c_uint32, _vp, _vp, _vp, C.c_uint32, C.POINTER(_DsgRes), _vp, _vp],
    "ga_core_exact_host": [C.c_uint32, _vp, _vp, C.c_uint64, _vp, _vp, C.c_int, C.POINTER(_DsgSeed),
                           C.POINTER(_DsgRes), _vp],
    "ga_exact_densest_host": [C.c_uint32, C.c_uint64, _vp, C.POINTER(_DsgRes), _vp],
    "ga_prune_to_core": [_vp, _vp, C.c_uint32, C.c_uint32, _vp, C.c_uint64, C.POINTER(C.POINTER(_HostGraph)), _vp,
                         _vp],
    "ga_gen_holme_kim_batch": [C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_double,
                               C.c_uint64, C.POINTER(C.POINTER(_HostBatch))],
    "ga_host_batch_free": [C.POINTER(_HostBatch)],
    "ga_batch_create": [C.c_uint32, _vp, _vp, _vp, _vp, C.c_int, _vp, C.POINTER(_vp)],
    "ga_batch_destroy": [_vp],
    "ga_batch_set_option": [_vp, C.c_int, C.c_int64],
    "ga_batch_device_bytes": [_vp, C.POINTER(C.c_uint64)],
    "ga_batch_tc": [_vp, _vp],
    "ga_batch_tc_peel": [_vp, C.c_uint64, C.c_uint64, _vp, _vp, _vp, _vp],
    "ga_server_create": [C.POINTER(_ServerConfig), C.POINTER(_vp)],
    "ga_server_destroy": [_vp],
    "ga_server_add_graph": [_vp, _u32p, _vp, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64)],
    "ga_server_submit": [_vp, C.c_uint64, C.c_int, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)],
    "ga_server_submit_out": [_vp, C.c_uint64, C.c_int, C.c_uint64, C.c_uint64, _vp, C.c_uint64,
                             C.POINTER(C.c_uint64)],
    "ga_server_poll": [_vp, C.c_uint64, C.POINTER(_RequestResult)],
    "ga_server_wait": [_vp, C.c_uint64, C.POINTER(_RequestResult)],
    "ga_server_stats_get": [_vp, C.POINTER(_ServerStats)],
}
_RESTYPE = {"ga_status_string": C.c_char_p, "ga_last_error": C.c_char_p, "ga_host_graph_free": None,
            "ga_host_batch_free": None}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Loads libga_b200.so (built by ``python -m graph_analyzer_b200.build``); raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built: run `python -m graph_analyzer_b200.build` "
                              "(the CUDA library is required; there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, C.c_int)
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status != 0:
        raise GAError(status, lib().ga_last_error().decode(errors="replace"))


def device_count() -> int:
    c = C.c_int(0)
    _check(lib().ga_device_count(C.byref(c)))
    return c.value


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


# ------------------------------------------------------------------------------------------------------------------
# graph.h surface
# ------------------------------------------------------------------------------------------------------------------

@dataclass
class Graph:
    """Oriented CSR, the fields of the reference's ``struct Graph`` (graph.h:19-26)."""

    n: int
    m: int
    rowptr: np.ndarray            # uint32[n+1]
    col: np.ndarray               # uint32[m], rows sorted
    src: np.ndarray               # uint32[m]
    max_out_degree: int

    def __eq__(self, other) -> bool:
        return (isinstance(other, Graph) and self.n == other.n and self.m == other.m
                and self.max_out_degree == other.max_out_degree and np.array_equal(self.rowptr, other.rowptr)
                and np.array_equal(self.col, other.col) and np.array_equal(self.src, other.src))


def canonical_edges(pairs: np.ndarray) -> np.ndarray:
    """load_graph's clean-up (graph.h:85-92): self loops dropped, (min,max), sorted, unique. Returns (k,2) uint32."""
    p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1).copy()
    if p.size == 0:
        return p.reshape(0, 2)
    k = C.c_uint64(0)
    _check(lib().ga_canonical_edges(p, p.size // 2, C.byref(k)))
    return p[: 2 * k.value].reshape(-1, 2)


def build_graph_from_edges(n: int, edges: np.ndarray) -> Graph:
    """build_graph_from_edges (graph.h:38-67): unique undirected pairs without self loops -> oriented CSR."""
    p = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1)
    m = p.size // 2
    rowptr = np.zeros(n + 1, np.uint32)
    col = np.zeros(max(m, 1), np.uint32)
    src = np.zeros(max(m, 1), np.uint32)
    mx = C.c_uint32(0)
    _check(lib().ga_build_graph_from_edges(n, p if m else np.zeros(2, np.uint32), m, rowptr, col, src,
                                           C.byref(mx)))
    return Graph(n, m, rowptr, col[:m].copy(), src[:m].copy(), mx.value)


def _from_host_graph(hg) -> Graph:
    h = hg.contents
    n, m = h.n, h.m
    rowptr = np.ctypeslib.as_array(h.rowptr, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(h.col, shape=(max(m, 1),))[:m].copy()
    src = np.ctypeslib.as_array(h.src, shape=(max(m, 1),))[:m].copy()
    g = Graph(n, m, rowptr, col, src, h.max_out_degree)
    lib().ga_host_graph_free(hg)
    return g


def load_graph(path: str) -> Graph:
    """load_graph (graph.h:71-96): SNAP text edge list -> cleaned, oriented CSR with n = max_id + 1."""
    hg = C.POINTER(_HostGraph)()
    _check(lib().ga_load_graph(os.fsencode(path), C.byref(hg)))
    return _from_host_graph(hg)


def save_csr(g: Graph, path: str) -> None:
    """Writes the oriented CSR as a binary file (checked first: sorted rows, ids < n, (degree, id) orientation)."""
    rowptr = np.ascontiguousarray(g.rowptr, np.uint32)
    col = np.ascontiguousarray(g.col, np.uint32)
    _check(lib().ga_save_csr(os.fsencode(path), g.n, g.m, rowptr, _ptr(col) if g.m else None))


def load_csr(path: str) -> Graph:
    """Reads a binary CSR file written by save_csr (header, size, checksum and CSR rules checked)."""
    hg = C.POINTER(_HostGraph)()
    _check(lib().ga_load_csr(os.fsencode(path), C.byref(hg)))
    return _from_host_graph(hg)


def graph_from_pairs(n: int, pairs: np.ndarray, canonicalize: bool = True) -> Graph:
    """Cleans (optionally) and orients an arbitrary undirected pair list on vertices 0..n-1."""
    p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1)
    hg = C.POINTER(_HostGraph)()
    _check(lib().ga_host_graph_from_edges(n, p if p.size else np.zeros(2, np.uint32), p.size // 2,
                                          int(canonicalize), C.byref(hg)))
    return _from_host_graph(hg)


# ------------------------------------------------------------------------------------------------------------------
# synthetic inputs
# ------------------------------------------------------------------------------------------------------------------

def gen_holme_kim(n: int, m_lo: int, m_hi: int | None = None, p_hi: float = 0.0, triad_p: float = 0.5,
                  seed: int = 1, permute: bool = True) -> np.ndarray:
    """Holme-Kim pairs (unique, no self loops), ids permuted from the seed. m_v = m_hi w.p. p_hi, else m_lo."""
    m_hi = m_lo if m_hi is None else m_hi
    cap = n * m_hi
    out = np.zeros(2 * max(cap, 1), np.uint32)
    k = C.c_uint64(0)
    _check(lib().ga_gen_holme_kim(n, m_lo, m_hi, p_hi, triad_p, seed, out, cap, C.byref(k)))
    pairs = out[: 2 * k.value]
    if permute:
        _check(lib().ga_permute_ids(pairs, k.value, n, seed))
    return pairs.reshape(-1, 2)


def gen_rmat(scale: int, nsamples: int, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
             permute: bool = True) -> np.ndarray:
    """Raw R-MAT samples on 2^scale vertices (clean with canonical_edges), ids permuted from the seed."""
    out = np.zeros(2 * max(nsamples, 1), np.uint32)
    _check(lib().ga_gen_rmat(scale, nsamples, a, b, c, seed, out))
    pairs = out[: 2 * nsamples]
    if permute:
        _check(lib().ga_permute_ids(pairs, nsamples, 1 << scale, seed))
    return pairs.reshape(-1, 2)


def permute_ids(pairs: np.ndarray, n: int, seed: int) -> np.ndarray:
    p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1).copy()
    _check(lib().ga_permute_ids(p, p.size // 2, n, seed))
    return p.reshape(-1, 2)


# ------------------------------------------------------------------------------------------------------------------
# densest.h helpers (integer arithmetic only; densest.h:62-78)
# ------------------------------------------------------------------------------------------------------------------

U64 = (1 << 64) - 1


def density_value(num: int, den: int) -> float:
    """Display value only (densest.h:62)."""
    return float(num) / float(den) if den else 0.0


def peel_arith_ok(n: int, T0: int, num: int, den: int) -> tuple[bool, str]:
    """peel_arith_ok (densest.h:65-72); returns (ok, why)."""
    if den < 1 or den > (1 << 20) or num > (1 << 20):
        return False, "eps = num/den needs 1 <= den <= 2^20 and num <= 2^20"
    if T0 >= (1 << 32):
        return False, "triangle count >= 2^32: uint32 tri[] counters could overflow"
    if n > 0 and T0 > U64 // (n * den):
        return False, "tri*nalive*den could overflow uint64"
    if T0 > U64 // (3 * (den + num)):
        return False, "3*(den+num)*T could overflow uint64"
    return True, ""


def peel_improves(T: int, nalive: int, best_num: int, best_den: int) -> bool:
    """peel_improves (densest.h:76-78): strict improvement; ties keep the earlier, larger set."""
    return best_den == 0 or T * best_den > best_num * nalive


@dataclass
class PeelResult:
    """PeelResult (densest.h:46-54); equality as operator== (densest.h:56-59)."""

    best_num: int = 0
    best_den: int = 0
    best_round: int = 0
    rounds: int = 0
    removed_round: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    ok: bool = True
    error: str = ""

    def __eq__(self, o) -> bool:
        return (self.best_num == o.best_num and self.best_den == o.best_den and self.best_round == o.best_round
                and self.rounds == o.rounds and np.array_equal(self.removed_round, o.removed_round))

    def density(self) -> float:
        return density_value(self.best_num, self.best_den)

    def peeled_set(self) -> np.ndarray:
        """{v : removed_round[v] >= best_round} (densest.h:13-14)."""
        return np.nonzero(self.removed_round >= self.best_round)[0].astype(np.uint32)


@dataclass
class DsgResult:
    """DsgResult (dsg.h:49-59): the returned vertex set (ascending ids) and its triangle count."""

    tri: int = 0
    verts: int = 0
    set: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    flow_calls: int = 0
    components_searched: int = 0
    shrinks: int = 0
    per_pass: list = field(default_factory=list)

    def density(self) -> float:
        return density_value(self.tri, self.verts)


def _dsg_result(r: _DsgRes, setbuf: np.ndarray, per: np.ndarray | None = None) -> DsgResult:
    pp = [(int(per[2 * i]), int(per[2 * i + 1])) for i in range(len(per) // 2)] if per is not None else []
    return DsgResult(r.tri, r.verts, setbuf[: r.verts].copy(), r.flow_calls, r.components_searched, r.shrinks, pp)


def _seed(seed: DsgResult | None):
    if seed is None:
        return None, None
    arr = np.ascontiguousarray(seed.set, np.uint32)
    return C.byref(_DsgSeed(_ptr(arr) if arr.size else None, arr.size, seed.tri, seed.verts)), arr


def greedy_pp_host(n: int, core: np.ndarray, inc_ptr: np.ndarray, inc: np.ndarray, passes: int) -> DsgResult:
    """Host stage of Greedy / Greedy++ on caller-made incidence lists (ga_greedy_pp_host)."""
    r, setbuf, per = _DsgRes(), np.zeros(max(n, 1), np.uint32), np.zeros(2 * max(passes, 1), np.uint64)
    core = np.ascontiguousarray(core, np.uint32)
    ip, ie = np.ascontiguousarray(inc_ptr, np.uint64), np.ascontiguousarray(inc, np.uint32)
    _check(lib().ga_greedy_pp_host(n, _ptr(core) if n else None, _ptr(ip), _ptr(ie) if ie.size else None, passes,
                                   C.byref(r), _ptr(setbuf), _ptr(per)))
    return _dsg_result(r, setbuf, per[: 2 * passes])


def core_exact_host(g: Graph, tris: np.ndarray, core: np.ndarray, use_pruning12: bool = True,
                    seed: DsgResult | None = None) -> DsgResult:
    """Host stage of CoreExact on caller-listed triangles (lowest, middle, highest) (ga_core_exact_host)."""
    r, setbuf = _DsgRes(), np.zeros(max(g.n, 1), np.uint32)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1)
    core = np.ascontiguousarray(core, np.uint32)
    sp, keep = _seed(seed)
    _check(lib().ga_core_exact_host(g.n, _ptr(np.ascontiguousarray(g.rowptr, np.uint32)),
                                    _ptr(np.ascontiguousarray(g.col, np.uint32)) if g.m else None, t.size // 3,
                                    _ptr(t) if t.size else None, _ptr(core) if g.n else None, int(use_pruning12), sp,
                                    C.byref(r), _ptr(setbuf)))
    del keep
    return _dsg_result(r, setbuf)


def exact_densest_host(n: int, tris: np.ndarray) -> DsgResult:
    r, setbuf = _DsgRes(), np.zeros(max(n, 1), np.uint32)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1)
    _check(lib().ga_exact_densest_host(n, t.size // 3, _ptr(t) if t.size else None, C.byref(r), _ptr(setbuf)))
    return _dsg_result(r, setbuf)


def prune_to_core(g: Graph, core: np.ndarray, k: int) -> tuple[Graph, np.ndarray, np.ndarray]:
    """prune_to_core (dsg.h:638-645): (subgraph of {core >= k}, old ids, restricted core numbers)."""
    out = C.POINTER(_HostGraph)()
    old, cout = np.zeros(max(g.n, 1), np.uint32), np.zeros(max(g.n, 1), np.uint32)
    core = np.ascontiguousarray(core, np.uint32)
    _check(lib().ga_prune_to_core(_ptr(np.ascontiguousarray(g.rowptr, np.uint32)),
                                  _ptr(np.ascontiguousarray(g.col, np.uint32)) if g.m else None, g.n, g.m,
                                  _ptr(core) if g.n else None, k, C.byref(out), _ptr(old), _ptr(cout)))
    gp = _from_host_graph(out)
    return gp, old[: gp.n].copy(), cout[: gp.n].copy()


@dataclass
class CoreResult:
    """Core numbers plus the CoreLoopResult fields (dsg.h:687-691)."""

    core: np.ndarray
    kmax: int
    rounds: int


# ------------------------------------------------------------------------------------------------------------------
# device-resident graph
# ------------------------------------------------------------------------------------------------------------------

class DeviceGraph:
    """A graph resident on one GPU (ga_graph). Use as a context manager or call close()."""

    def __init__(self, g: Graph, device: int = 0, stream: int | None = None):
        self.n, self.m = g.n, g.m
        h = _vp()
        rowptr = np.ascontiguousarray(g.rowptr, np.uint32)
        col = np.ascontiguousarray(g.col if g.m else np.zeros(1, np.uint32), np.uint32)
        _check(lib().ga_graph_create(_ptr(rowptr), _ptr(col), g.n, g.m, device, stream, C.byref(h)))
        self._h = h

    @classmethod
    def from_device(cls, d_rowptr: int, d_col: int, n: int, m: int, device: int = 0, stream: int | None = None):
        self = cls.__new__(cls)
        self.n, self.m = n, m
        h = _vp()
        _check(lib().ga_graph_create_device(d_rowptr, d_col, n, m, device, stream, C.byref(h)))
        self._h = h
        return self

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().ga_graph_destroy(self._h)
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, opt: int, value: int) -> None:
        _check(lib().ga_graph_set_option(self._h, opt, value))

    def set_stream(self, stream: int | None) -> None:
        _check(lib().ga_graph_set_stream(self._h, stream))

    def prepare(self) -> None:
        _check(lib().ga_graph_prepare(self._h))

    def device_bytes(self) -> int:
        b = C.c_uint64(0)
        _check(lib().ga_graph_device_bytes(self._h, C.byref(b)))
        return b.value

    def tc_count(self) -> int:
        t = C.c_uint64(0)
        _check(lib().ga_tc_count(self._h, C.byref(t)))
        return t.value

    def tc_count_shard(self, shard: int, nshards: int) -> int:
        """Triangles of shard `shard` of `nshards`; the shards' sum is tc_count()."""
        t = C.c_uint64(0)
        _check(lib().ga_tc_count_shard(self._h, shard, nshards, C.byref(t)))
        return t.value

    def tc_count_shard_async(self, shard: int, nshards: int, d_out: int) -> None:
        _check(lib().ga_tc_count_shard_async(self._h, shard, nshards, d_out))

    def tc_count_async(self, d_out: int) -> None:
        """Enqueues the count on the graph's stream; the result lands in 8 bytes of device memory at d_out."""
        _check(lib().ga_tc_count_async(self._h, d_out))

    def support_edges(self) -> tuple[int, np.ndarray]:
        sup = np.zeros(max(self.m, 1), np.uint32)
        t = C.c_uint64(0)
        _check(lib().ga_tc_support_edges(self._h, _ptr(sup), C.byref(t)))
        return t.value, sup[: self.m]

    def support_edges_device(self, d_sup: int) -> int:
        t = C.c_uint64(0)
        _check(lib().ga_tc_support_edges_device(self._h, d_sup, C.byref(t)))
        return t.value

    def support_vertices(self) -> tuple[int, np.ndarray]:
        deg = np.zeros(max(self.n, 1), np.uint64)
        t = C.c_uint64(0)
        _check(lib().ga_tc_support_vertices(self._h, _ptr(deg), C.byref(t)))
        return t.value, deg[: self.n]

    def participation(self, alive: np.ndarray) -> tuple[int, np.ndarray]:
        a = np.ascontiguousarray(alive, np.uint8)
        if a.size != self.n:
            raise ValueError("alive must have n entries")
        tri = np.zeros(max(self.n, 1), np.uint32)
        t = C.c_uint64(0)
        _check(lib().ga_tc_participation(self._h, _ptr(a if self.n else np.zeros(1, np.uint8)), _ptr(tri),
                                         C.byref(t)))
        return t.value, tri[: self.n]

    def tuning(self) -> dict:
        """The count configuration (kernel, bin cutoff, item work) the autotuner chose for this graph."""
        t = _Tuning()
        _check(lib().ga_graph_tuning(self._h, C.byref(t)))
        return _tuning_dict(t)

    def core_level_density(self, core: np.ndarray, k: int) -> tuple[int, int]:
        """(triangles, vertices) of {v : core[v] >= k} (core_level_density, dsg.h:169-174)."""
        c = np.ascontiguousarray(core, np.uint32)
        if c.size != self.n:
            raise ValueError("core must have n entries")
        t, v = C.c_uint64(0), C.c_uint64(0)
        _check(lib().ga_core_level_density(self._h, _ptr(c if self.n else np.zeros(1, np.uint32)), k, C.byref(t),
                                           C.byref(v)))
        return t.value, v.value

    def batch_peel(self, num: int = 1, den: int = 10, want_removed: bool = True) -> PeelResult:
        r = _PeelRes()
        rr = np.full(max(self.n, 1), 0xFFFFFFFF, np.uint32) if want_removed else None
        _check(lib().ga_batch_peel(self._h, num, den, C.byref(r), _ptr(rr)))
        return PeelResult(r.best_num, r.best_den, r.best_round, r.rounds,
                          rr[: self.n] if rr is not None else np.zeros(0, np.uint32))

    def core_decomposition(self, want_core: bool = True) -> CoreResult:
        r = _CoreRes()
        core = np.zeros(max(self.n, 1), np.uint32) if want_core else None
        _check(lib().ga_core_decomposition(self._h, _ptr(core), C.byref(r)))
        return CoreResult(core[: self.n] if core is not None else np.zeros(0, np.uint32), r.kmax, r.rounds)


    def greedy_pp(self, passes: int = 1) -> DsgResult:
        """Greedy (passes = 1) / Greedy++ (dsg.h:189-250): core numbers and triangle lists on the device."""
        r, setbuf = _DsgRes(), np.zeros(max(self.n, 1), np.uint32)
        per = np.zeros(2 * max(passes, 1), np.uint64)
        _check(lib().ga_greedy_pp(self._h, passes, C.byref(r), _ptr(setbuf), _ptr(per)))
        return _dsg_result(r, setbuf, per[: 2 * passes])

    def core_exact(self, core: np.ndarray | None = None, use_pruning12: bool = True,
                   seed: DsgResult | None = None) -> DsgResult:
        """CoreExact (dsg.h:463-627); core numbers from the device when `core` is None."""
        r, setbuf = _DsgRes(), np.zeros(max(self.n, 1), np.uint32)
        if core is not None and len(core) != self.n:
            raise ValueError("core must have n entries")
        c = np.ascontiguousarray(core, np.uint32) if core is not None and self.n else None
        sp, keep = _seed(seed)
        _check(lib().ga_core_exact(self._h, _ptr(c), int(use_pruning12), sp, C.byref(r), _ptr(setbuf)))
        del keep
        return _dsg_result(r, setbuf)

    def exact_densest(self) -> DsgResult:
        """Exact (dsg.h:405-428)."""
        r, setbuf = _DsgRes(), np.zeros(max(self.n, 1), np.uint32)
        _check(lib().ga_exact_densest(self._h, C.byref(r), _ptr(setbuf)))
        return _dsg_result(r, setbuf)


# one-shot helpers with the reference driver's semantics (upload, run, download)

def gpu_triangles(g: Graph, device: int = 0) -> int:
    with DeviceGraph(g, device) as d:
        return d.tc_count()


def gpu_batch_peel(g: Graph, num: int = 1, den: int = 10, device: int = 0) -> PeelResult:
    with DeviceGraph(g, device) as d:
        return d.batch_peel(num, den)


def gpu_core_decomposition(g: Graph, device: int = 0) -> CoreResult:
    with DeviceGraph(g, device) as d:
        return d.core_decomposition()


# ------------------------------------------------------------------------------------------------------------------
# batches: many graphs packed as one concatenated CSR (64-bit offsets, 32-bit local ids)
# ------------------------------------------------------------------------------------------------------------------

@dataclass
class HostBatch:
    """Packed batch: graph i owns vertices [vtx_off[i], vtx_off[i+1]) and edges [edge_off[i], edge_off[i+1]); its
    local rowptr (n_i + 1 entries) starts at rowptr[vtx_off[i] + i]; col holds local ids."""

    vtx_off: np.ndarray   # uint64[G+1]
    edge_off: np.ndarray  # uint64[G+1]
    rowptr: np.ndarray    # uint32[N+G]
    col: np.ndarray       # uint32[M]

    @property
    def num_graphs(self) -> int:
        return len(self.vtx_off) - 1

    def graph(self, i: int) -> Graph:
        v0, v1 = int(self.vtx_off[i]), int(self.vtx_off[i + 1])
        e0, e1 = int(self.edge_off[i]), int(self.edge_off[i + 1])
        rowptr = self.rowptr[v0 + i: v1 + i + 1].copy()
        col = self.col[e0:e1].copy()
        d = np.diff(rowptr.astype(np.int64))
        src = np.repeat(np.arange(v1 - v0, dtype=np.uint32), d)
        return Graph(v1 - v0, e1 - e0, rowptr, col, src, int(d.max()) if d.size else 0)


def pack_batch(graphs: list[Graph]) -> HostBatch:
    vtx_off = np.zeros(len(graphs) + 1, np.uint64)
    edge_off = np.zeros(len(graphs) + 1, np.uint64)
    vtx_off[1:] = np.cumsum([g.n for g in graphs])
    edge_off[1:] = np.cumsum([g.m for g in graphs])
    rowptr = np.concatenate([g.rowptr for g in graphs]).astype(np.uint32)
    col = (np.concatenate([g.col for g in graphs]) if graphs else np.zeros(0)).astype(np.uint32)
    return HostBatch(vtx_off, edge_off, rowptr, col)


def gen_holme_kim_batch(num_graphs: int, n_lo: int = 64, n_hi: int = 262144, deg_lo: float = 4.0,
                        deg_hi: float = 32.0, p_lo: float = 0.1, p_hi: float = 0.7, seed: int = 1) -> HostBatch:
    """Seeded batch of Holme-Kim graphs (n log-uniform, mean degree and triad probability uniform), built in
    parallel on the host."""
    hb = C.POINTER(_HostBatch)()
    _check(lib().ga_gen_holme_kim_batch(num_graphs, n_lo, n_hi, deg_lo, deg_hi, p_lo, p_hi, seed, C.byref(hb)))
    h = hb.contents
    G, N, M = h.num_graphs, h.total_vertices, h.total_edges
    out = HostBatch(np.ctypeslib.as_array(h.vtx_off, shape=(G + 1,)).copy(),
                    np.ctypeslib.as_array(h.edge_off, shape=(G + 1,)).copy(),
                    np.ctypeslib.as_array(h.rowptr, shape=(N + G,)).copy(),
                    np.ctypeslib.as_array(h.col, shape=(max(M, 1),))[:M].copy())
    lib().ga_host_batch_free(hb)
    return out


@dataclass
class BatchPeel:
    triangles: np.ndarray       # uint64[G]
    best_num: np.ndarray        # uint64[G]
    best_den: np.ndarray        # uint64[G]
    best_round: np.ndarray      # uint32[G]
    rounds: np.ndarray          # uint32[G]
    status: np.ndarray          # uint32[G] (ga_status per graph)
    removed_round: np.ndarray   # uint32[N], batch order

    def result(self, batch: HostBatch, i: int) -> PeelResult:
        v0, v1 = int(batch.vtx_off[i]), int(batch.vtx_off[i + 1])
        return PeelResult(int(self.best_num[i]), int(self.best_den[i]), int(self.best_round[i]),
                          int(self.rounds[i]), self.removed_round[v0:v1])


class DeviceBatch:
    """A packed batch resident on one GPU (ga_batch)."""

    def __init__(self, b: HostBatch, device: int = 0, stream: int | None = None):
        self.G = b.num_graphs
        self.N = int(b.vtx_off[-1])
        vo = np.ascontiguousarray(b.vtx_off, np.uint64)
        eo = np.ascontiguousarray(b.edge_off, np.uint64)
        rp = np.ascontiguousarray(b.rowptr, np.uint32)
        cl = np.ascontiguousarray(b.col if b.col.size else np.zeros(1, np.uint32), np.uint32)
        h = _vp()
        _check(lib().ga_batch_create(self.G, _ptr(vo), _ptr(eo), _ptr(rp), _ptr(cl), device, stream, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().ga_batch_destroy(self._h)
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, opt: int, value: int) -> None:
        _check(lib().ga_batch_set_option(self._h, opt, value))

    def device_bytes(self) -> int:
        b = C.c_uint64(0)
        _check(lib().ga_batch_device_bytes(self._h, C.byref(b)))
        return b.value

    def tuning(self) -> dict:
        """The count configuration of the batch's launch over the union of its graphs."""
        t = _Tuning()
        _check(lib().ga_batch_tuning(self._h, C.byref(t)))
        return _tuning_dict(t)

    def tc(self) -> np.ndarray:
        t = np.zeros(self.G, np.uint64)
        _check(lib().ga_batch_tc(self._h, _ptr(t)))
        return t

    def tc_peel(self, num: int = 1, den: int = 10, want_removed: bool = True) -> BatchPeel:
        G = self.G
        t = np.zeros(G, np.uint64)
        res = (_PeelRes * G)()
        st = np.zeros(G, np.uint32)
        rr = np.zeros(max(self.N, 1), np.uint32) if want_removed else None
        _check(lib().ga_batch_tc_peel(self._h, num, den, _ptr(t), C.addressof(res), _ptr(st), _ptr(rr)))
        return BatchPeel(t, np.array([r.best_num for r in res], np.uint64),
                         np.array([r.best_den for r in res], np.uint64),
                         np.array([r.best_round for r in res], np.uint32),
                         np.array([r.rounds for r in res], np.uint32), st,
                         rr[: self.N] if rr is not None else np.zeros(0, np.uint32))


# ------------------------------------------------------------------------------------------------------------------
# serving: request loop with admission by HBM budget, resident graphs and folded batch launches (ga_server)
# ------------------------------------------------------------------------------------------------------------------

REQ_TC, REQ_PEEL, REQ_CORE = 0, 1, 2
GA_ERR_NOT_READY = 12


@dataclass
class RequestResult:
    status: int
    triangles: int
    peel: PeelResult            # REQ_PEEL (removed_round filled when the request was submitted with want_array)
    core: tuple[int, int]       # REQ_CORE: (kmax, rounds)
    queue_ms: float
    run_ms: float
    folded: int                 # graphs served by the same launch (1 = alone)
    resident_hit: bool
    core_numbers: np.ndarray | None = None   # REQ_CORE submitted with want_array: core[v] for every vertex


def _request_result(r: _RequestResult) -> RequestResult:
    return RequestResult(r.status, r.triangles,
                         PeelResult(r.peel.best_num, r.peel.best_den, r.peel.best_round, r.peel.rounds),
                         (r.core.kmax, r.core.rounds), r.queue_ms, r.run_ms, r.folded, bool(r.resident_hit))


class Server:
    """A request loop on one GPU (ga_server): graphs are registered once, requests are submitted without waiting and
    run concurrently on `slots` streams; small count/peel requests queued together share one batch launch."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, slots: int = 0, fold_max_graphs: int = 0,
                 fold_max_edges: int = 0, small_slots: int = 0, pin_min_edges: int = 0):
        cfg = _ServerConfig(device, hbm_budget_bytes, slots, fold_max_graphs, fold_max_edges, small_slots,
                            pin_min_edges)
        h = _vp()
        self._n: dict[int, int] = {}                      # vertices per registered graph
        self._arrays: dict[int, tuple] = {}               # ticket -> (kind, host array the server writes, n)
        _check(lib().ga_server_create(C.byref(cfg), C.byref(h)))
        self._h = h

    def close(self) -> None:
        """Waits for every submitted request, then frees the device memory."""
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().ga_server_destroy(self._h)
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_graph(self, g: Graph) -> int:
        gid = C.c_uint64(0)
        rowptr = np.ascontiguousarray(g.rowptr, np.uint32)
        col = np.ascontiguousarray(g.col, np.uint32)
        _check(lib().ga_server_add_graph(self._h, rowptr, _ptr(col) if g.m else None, g.n, g.m, C.byref(gid)))
        self._n[gid.value] = g.n
        return gid.value

    def submit(self, graph_id: int, kind: int, num: int = 1, den: int = 10, want_array: bool = False) -> int:
        """Queues a request. want_array: also return the vertex array (removed_round of a peel, core numbers of a
        core decomposition) in the result."""
        t = C.c_uint64(0)
        if want_array and kind != REQ_TC:
            n = self._n[graph_id]
            buf = np.full(max(n, 1), 0xFFFFFFFF, np.uint32)
            _check(lib().ga_server_submit_out(self._h, graph_id, kind, num, den, _ptr(buf), buf.size, C.byref(t)))
            self._arrays[t.value] = (kind, buf, n)     # kept alive until the result is collected
        else:
            _check(lib().ga_server_submit(self._h, graph_id, kind, num, den, C.byref(t)))
        return t.value

    def _result(self, ticket: int, r: _RequestResult) -> RequestResult:
        res = _request_result(r)
        kind_buf = self._arrays.pop(ticket, None)
        if kind_buf is not None:
            kind, buf, n = kind_buf
            if kind == REQ_PEEL:
                res.peel.removed_round = buf[:n]
            else:
                res.core_numbers = buf[:n]
        return res

    def poll(self, ticket: int) -> RequestResult | None:
        r = _RequestResult()
        st = lib().ga_server_poll(self._h, ticket, C.byref(r))
        if st == GA_ERR_NOT_READY:
            return None
        _check(st)
        return self._result(ticket, r)

    def wait_for(self, ticket: int, timeout_s: float) -> RequestResult | None:
        """The result of `ticket` once ready, or None after `timeout_s` seconds (the request stays pending)."""
        t_end = time.monotonic() + timeout_s
        while True:
            r = self.poll(ticket)
            if r is not None or time.monotonic() >= t_end:
                return r
            time.sleep(0.01)

    def wait(self, ticket: int) -> RequestResult:
        r = _RequestResult()
        _check(lib().ga_server_wait(self._h, ticket, C.byref(r)))
        return self._result(ticket, r)

    def stats(self) -> dict:
        st = _ServerStats()
        _check(lib().ga_server_stats_get(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _ServerStats._fields_}
