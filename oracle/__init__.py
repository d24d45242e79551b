"""numpy bindings of the checker libraries (TEST INFRASTRUCTURE).

``Oracle`` wraps oracle/liboracle.so (the plain-C restatement in ga_oracle.c); ``Reference`` wraps
oracle/_ref/libga_ref.so (the reference's own CPU code compiled from its headers). Both expose the same method names
so a test can run one against the other. Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this package; the product (graph_analyzer_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import build_oracle

HERE = os.path.dirname(os.path.abspath(__file__))

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


@dataclass
class CSR:
    """Oriented CSR with the fields of the reference's Graph (graph.h:19-26)."""

    n: int
    m: int
    rowptr: np.ndarray
    col: np.ndarray
    src: np.ndarray
    max_out_degree: int


@dataclass
class PeelOut:
    best_num: int
    best_den: int
    best_round: int
    rounds: int
    ok: bool
    removed_round: np.ndarray


@dataclass
class DsgOut:
    """DsgResult of dsg.h: the returned vertex set (ascending ids) with its triangle count."""
    tri: int
    verts: int
    set: np.ndarray
    flow_calls: int = 0
    components_searched: int = 0
    shrinks: int = 0
    per_pass: list | None = None


class _Base:
    lib: C.CDLL

    def _args(self, g: CSR):
        return (g.n, g.m, g.rowptr, g.col, g.src)


class Oracle(_Base):
    """Plain-C restatement; every method cites the reference function it restates (see ga_oracle.h)."""

    def __init__(self, path: str | None = None):
        path = path or build_oracle.build_oracle()
        L = self.lib = C.CDLL(path)
        L.or_canonical_edges.restype = C.c_uint64
        L.or_canonical_edges.argtypes = [_u32p, C.c_uint64]
        L.or_build_graph.restype = C.c_int
        L.or_build_graph.argtypes = [C.c_uint32, _u32p, C.c_uint32, _u32p, _u32p, _u32p, C.POINTER(C.c_uint32)]
        L.or_count_text_pairs.restype = C.c_int64
        L.or_count_text_pairs.argtypes = [C.c_char_p]
        L.or_read_text_pairs.restype = C.c_int64
        L.or_read_text_pairs.argtypes = [C.c_char_p, _u32p, C.c_uint64, C.POINTER(C.c_uint32)]
        L.or_triangles_serial.restype = C.c_uint64
        L.or_triangles_serial.argtypes = [C.c_uint32, _u32p, _u32p]
        L.or_triangles_omp.restype = C.c_uint64
        L.or_triangles_omp.argtypes = [C.c_uint32, _u32p, _u32p]
        L.or_num_threads.restype = C.c_int
        L.or_participation.restype = C.c_uint64
        L.or_participation.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u8p, _u32p]
        L.or_edge_support.restype = C.c_uint64
        L.or_edge_support.argtypes = [C.c_uint32, _u32p, _u32p, _u32p, _u32p]
        L.or_edge_support_omp.restype = C.c_uint64
        L.or_edge_support_omp.argtypes = [C.c_uint32, _u32p, _u32p, _u32p, _u32p]
        L.or_triangle_degrees.restype = C.c_uint64
        L.or_triangle_degrees.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u64p]
        L.or_peel_arith_ok.restype = C.c_int
        L.or_peel_arith_ok.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64]
        L.or_peel_improves.restype = C.c_int
        L.or_peel_improves.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]
        L.or_batch_peel.restype = None
        L.or_batch_peel.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, C.c_uint64, C.c_uint64,
                                    C.c_void_p, _u32p]
        L.or_undirected_csr.restype = None
        L.or_undirected_csr.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p]
        L.or_core_decomposition.restype = C.c_int
        L.or_core_decomposition.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p,
                                            C.POINTER(C.c_uint32)]
        L.or_core_levels.restype = C.c_int
        L.or_core_levels.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p, C.POINTER(C.c_uint32),
                                     C.POINTER(C.c_uint32)]
        L.or_core_levels_inc.restype = C.c_int
        L.or_core_levels_inc.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p, C.POINTER(C.c_uint32),
                                         C.POINTER(C.c_uint32)]
        L.or_core_level_density.restype = None
        L.or_core_level_density.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p, C.c_uint32,
                                            C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.or_greedy_pp.restype = C.c_int
        L.or_greedy_pp.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, C.c_uint32, C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint64), _u32p, _u64p]

    # graph.h
    def canonical_edges(self, pairs: np.ndarray) -> np.ndarray:
        p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1).copy()
        k = self.lib.or_canonical_edges(p, len(p) // 2)
        return p[: 2 * k].reshape(-1, 2)

    def build_graph_from_edges(self, n: int, pairs: np.ndarray) -> CSR:
        p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1)
        m = len(p) // 2
        rowptr = np.zeros(n + 1, np.uint32)
        col = np.zeros(max(m, 1), np.uint32)
        src = np.zeros(max(m, 1), np.uint32)
        mx = C.c_uint32(0)
        if self.lib.or_build_graph(n, p if m else np.zeros(2, np.uint32), m, rowptr, col, src, C.byref(mx)) != 0:
            raise ValueError("edge endpoint >= n")
        return CSR(n, m, rowptr, col[:m].copy(), src[:m].copy(), int(mx.value))

    def load_graph(self, path: str) -> CSR:
        cnt = self.lib.or_count_text_pairs(path.encode())
        if cnt < 0:
            raise OSError(f"cannot open {path}")
        pairs = np.zeros(2 * max(cnt, 1), np.uint32)
        n = C.c_uint32(0)
        self.lib.or_read_text_pairs(path.encode(), pairs, cnt, C.byref(n))
        k = self.lib.or_canonical_edges(pairs, cnt)
        return self.build_graph_from_edges(int(n.value), pairs[: 2 * k])

    def triangles_serial(self, g: CSR) -> int:
        return int(self.lib.or_triangles_serial(g.n, g.rowptr, _col(g)))

    def triangles_omp(self, g: CSR) -> int:
        return int(self.lib.or_triangles_omp(g.n, g.rowptr, _col(g)))

    def num_threads(self) -> int:
        return int(self.lib.or_num_threads())

    # densest.h / dsg.h
    def participation(self, g: CSR, alive: np.ndarray) -> tuple[int, np.ndarray]:
        tri = np.zeros(max(g.n, 1), np.uint32)
        T = self.lib.or_participation(g.n, g.m, g.rowptr, _col(g), _src(g), _alive(alive, g.n), tri)
        return int(T), tri[: g.n]

    def edge_support(self, g: CSR, use_omp: bool = False) -> tuple[int, np.ndarray]:
        sup = np.zeros(max(g.m, 1), np.uint32)
        f = self.lib.or_edge_support_omp if use_omp else self.lib.or_edge_support
        T = f(g.m, g.rowptr, _col(g), _src(g), sup)
        return int(T), sup[: g.m]

    def triangle_degrees(self, g: CSR) -> tuple[int, np.ndarray]:
        deg = np.zeros(max(g.n, 1), np.uint64)
        T = self.lib.or_triangle_degrees(g.n, g.m, g.rowptr, _col(g), _src(g), deg)
        return int(T), deg[: g.n]

    def peel_arith_ok(self, n, T0, num, den) -> bool:
        return bool(self.lib.or_peel_arith_ok(n, T0, num, den))

    def peel_improves(self, T, nalive, bn, bd) -> bool:
        return bool(self.lib.or_peel_improves(T, nalive, bn, bd))

    def batch_peel(self, g: CSR, num: int, den: int) -> PeelOut:
        class R(C.Structure):
            _fields_ = [("best_num", C.c_uint64), ("best_den", C.c_uint64), ("best_round", C.c_uint32),
                        ("rounds", C.c_uint32), ("ok", C.c_int)]
        r = R()
        rr = np.zeros(max(g.n, 1), np.uint32)
        self.lib.or_batch_peel(g.n, g.m, g.rowptr, _col(g), _src(g), num, den, C.addressof(r), rr)
        return PeelOut(r.best_num, r.best_den, r.best_round, r.rounds, bool(r.ok), rr[: g.n])

    def undirected_csr(self, g: CSR) -> tuple[np.ndarray, np.ndarray]:
        urow = np.zeros(g.n + 1, np.uint32)
        ucol = np.zeros(max(2 * g.m, 1), np.uint32)
        self.lib.or_undirected_csr(g.n, g.m, _col(g), _src(g), urow, ucol)
        return urow, ucol[: 2 * g.m]

    def core_decomposition(self, g: CSR) -> tuple[np.ndarray, int]:
        core = np.zeros(max(g.n, 1), np.uint32)
        k = C.c_uint32(0)
        if self.lib.or_core_decomposition(g.n, g.m, g.rowptr, _col(g), _src(g), core, C.byref(k)) != 0:
            raise OverflowError("core number does not fit uint32")
        return core[: g.n], int(k.value)

    def core_levels(self, g: CSR) -> tuple[np.ndarray, int, int]:
        core = np.zeros(max(g.n, 1), np.uint32)
        k, r = C.c_uint32(0), C.c_uint32(0)
        if self.lib.or_core_levels(g.n, g.m, g.rowptr, _col(g), _src(g), core, C.byref(k), C.byref(r)) != 0:
            raise OverflowError("triangle count >= 2^32")
        return core[: g.n], int(k.value), int(r.value)

    def core_levels_inc(self, g: CSR) -> tuple[np.ndarray, int, int]:
        """Same as core_levels (core[], kmax, level rounds) by the incremental frontier loop: O(T) updates."""
        core = np.zeros(max(g.n, 1), np.uint32)
        k, r = C.c_uint32(0), C.c_uint32(0)
        rc = self.lib.or_core_levels_inc(g.n, g.m, g.rowptr, _col(g), _src(g), core, C.byref(k), C.byref(r))
        if rc == -1:
            raise OverflowError("triangle count >= 2^32")
        if rc != 0:
            raise MemoryError("or_core_levels_inc: out of host memory")
        return core[: g.n], int(k.value), int(r.value)

    def core_level_density(self, g: CSR, core: np.ndarray, k: int) -> tuple[int, int]:
        a, b = C.c_uint64(0), C.c_uint64(0)
        c = np.ascontiguousarray(core, np.uint32) if g.n else np.zeros(1, np.uint32)
        self.lib.or_core_level_density(g.n, g.m, g.rowptr, _col(g), _src(g), c, k, C.byref(a), C.byref(b))
        return int(a.value), int(b.value)

    def greedy_pp(self, g: CSR, passes: int) -> DsgOut:
        a, b = C.c_uint64(0), C.c_uint64(0)
        setbuf, per = np.zeros(max(g.n, 1), np.uint32), np.zeros(2 * max(passes, 1), np.uint64)
        if self.lib.or_greedy_pp(g.n, g.m, g.rowptr, _col(g), _src(g), passes, C.byref(a), C.byref(b), setbuf, per):
            raise RuntimeError("greedy_pp: triangle bookkeeping inconsistent")
        return DsgOut(int(a.value), int(b.value), setbuf[: int(b.value)].copy(),
                      per_pass=[(int(per[2 * i]), int(per[2 * i + 1])) for i in range(passes)])


class Reference(_Base):
    """The reference's own CPU code (oracle/_ref/libga_ref.so), same method names as ``Oracle``."""

    def __init__(self, path: str | None = None):
        path = path or build_oracle.build_ref()
        if not path or not os.path.exists(path):
            raise FileNotFoundError("oracle/_ref/libga_ref.so is not built (reference sources absent)")
        L = self.lib = C.CDLL(path)
        L.ref_build_graph.restype = C.c_int
        L.ref_build_graph.argtypes = [C.c_uint32, _u32p, C.c_uint32, _u32p, _u32p, _u32p, C.POINTER(C.c_uint32)]
        L.ref_load_graph_sizes.restype = C.c_int
        L.ref_load_graph_sizes.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.ref_load_graph.restype = C.c_int
        L.ref_load_graph.argtypes = [C.c_char_p, _u32p, _u32p, _u32p, C.POINTER(C.c_uint32)]
        for f in ("ref_triangles_serial", "ref_triangles_omp"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p]
        L.ref_num_threads.restype = C.c_int
        L.ref_graph_new.restype = C.c_void_p
        L.ref_graph_new.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p]
        L.ref_graph_free.restype = None
        L.ref_graph_free.argtypes = [C.c_void_p]
        L.ref_graph_triangles_omp.restype = C.c_uint64
        L.ref_graph_triangles_omp.argtypes = [C.c_void_p]
        L.ref_graph_triangles_omp_rows.restype = C.c_uint64
        L.ref_graph_triangles_omp_rows.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        L.ref_graph_triangles_serial_rows.restype = C.c_uint64
        L.ref_graph_triangles_serial_rows.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        L.ref_participation.restype = C.c_uint64
        L.ref_participation.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u8p, _u32p, C.c_int]
        L.ref_edge_support.restype = C.c_uint64
        L.ref_edge_support.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p]
        L.ref_triangle_degrees.restype = C.c_uint64
        L.ref_triangle_degrees.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u64p]
        L.ref_peel_arith_ok.restype = C.c_int
        L.ref_peel_arith_ok.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64]
        L.ref_peel_improves.restype = C.c_int
        L.ref_peel_improves.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]
        L.ref_batch_peel.restype = C.c_int
        L.ref_batch_peel.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, C.c_uint64, C.c_uint64, C.c_int,
                                     _u64p, _u32p]
        L.ref_undirected_csr.restype = None
        L.ref_undirected_csr.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p, _u32p]
        L.ref_core_decomposition.restype = C.c_int
        L.ref_core_decomposition.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p,
                                             C.POINTER(C.c_uint32)]
        L.ref_core_levels.restype = C.c_int
        L.ref_core_levels.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p, C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint32)]
        L.ref_core_level_density.restype = None
        L.ref_core_level_density.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p, _u32p, C.c_uint32,
                                             C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]

        _g = [C.c_uint32, C.c_uint32, _u32p, _u32p, _u32p]
        L.ref_greedy_pp.restype = C.c_int
        L.ref_greedy_pp.argtypes = _g + [C.c_uint32, _u64p, _u32p, _u64p, C.c_char_p, C.c_int]
        L.ref_cpu_greedy_peel.restype = C.c_int
        L.ref_cpu_greedy_peel.argtypes = _g + [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.ref_core_exact.restype = C.c_int
        L.ref_core_exact.argtypes = _g + [_u32p, C.c_int, C.c_int, _u32p, C.c_uint64, C.c_uint64, C.c_uint64, _u64p,
                                          _u32p, C.c_char_p, C.c_int]
        L.ref_exact_densest.restype = C.c_int
        L.ref_exact_densest.argtypes = _g + [_u64p, _u32p, C.c_char_p, C.c_int]
        L.ref_prune_to_core.restype = None
        L.ref_prune_to_core.argtypes = _g + [_u32p, C.c_uint64, _u32p, _u32p, _u32p, _u32p, _u32p,
                                             C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]

    def resident(self, g: CSR) -> "RefGraph":
        """A copy of g held in the reference's own Graph, for timing its counter without the copy-in."""
        return RefGraph(self, g)

    def build_graph_from_edges(self, n: int, pairs: np.ndarray) -> CSR:
        p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1)
        m = len(p) // 2
        rowptr = np.zeros(n + 1, np.uint32)
        col = np.zeros(max(m, 1), np.uint32)
        src = np.zeros(max(m, 1), np.uint32)
        mx = C.c_uint32(0)
        self.lib.ref_build_graph(n, p if m else np.zeros(2, np.uint32), m, rowptr, col, src, C.byref(mx))
        return CSR(n, m, rowptr, col[:m].copy(), src[:m].copy(), int(mx.value))

    def load_graph(self, path: str) -> CSR:
        n, m = C.c_uint32(0), C.c_uint32(0)
        if self.lib.ref_load_graph_sizes(path.encode(), C.byref(n), C.byref(m)) != 0:
            raise OSError(f"cannot open {path}")
        n, m = int(n.value), int(m.value)
        rowptr = np.zeros(n + 1, np.uint32)
        col = np.zeros(max(m, 1), np.uint32)
        src = np.zeros(max(m, 1), np.uint32)
        mx = C.c_uint32(0)
        self.lib.ref_load_graph(path.encode(), rowptr, col, src, C.byref(mx))
        return CSR(n, m, rowptr, col[:m].copy(), src[:m].copy(), int(mx.value))

    def triangles_serial(self, g: CSR) -> int:
        return int(self.lib.ref_triangles_serial(*self._args2(g)))

    def triangles_omp(self, g: CSR) -> int:
        return int(self.lib.ref_triangles_omp(*self._args2(g)))

    def num_threads(self) -> int:
        return int(self.lib.ref_num_threads())

    def _args2(self, g: CSR):
        return (g.n, g.m, g.rowptr, _col(g), _src(g))

    def participation(self, g: CSR, alive: np.ndarray, use_omp: bool = False) -> tuple[int, np.ndarray]:
        tri = np.zeros(max(g.n, 1), np.uint32)
        T = self.lib.ref_participation(*self._args2(g), _alive(alive, g.n), tri, int(use_omp))
        return int(T), tri[: g.n]

    def edge_support(self, g: CSR) -> tuple[int, np.ndarray]:
        sup = np.zeros(max(g.m, 1), np.uint32)
        T = self.lib.ref_edge_support(*self._args2(g), sup)
        return int(T), sup[: g.m]

    def triangle_degrees(self, g: CSR) -> tuple[int, np.ndarray]:
        deg = np.zeros(max(g.n, 1), np.uint64)
        T = self.lib.ref_triangle_degrees(*self._args2(g), deg)
        return int(T), deg[: g.n]

    def peel_arith_ok(self, n, T0, num, den) -> bool:
        return bool(self.lib.ref_peel_arith_ok(n, T0, num, den))

    def peel_improves(self, T, nalive, bn, bd) -> bool:
        return bool(self.lib.ref_peel_improves(T, nalive, bn, bd))

    def batch_peel(self, g: CSR, num: int, den: int, use_omp: bool = False) -> PeelOut:
        out = np.zeros(4, np.uint64)
        rr = np.full(max(g.n, 1), 0xFFFFFFFF, np.uint32)
        ok = self.lib.ref_batch_peel(*self._args2(g), num, den, int(use_omp), out, rr)
        return PeelOut(int(out[0]), int(out[1]), int(out[2]), int(out[3]), bool(ok), rr[: g.n])

    def undirected_csr(self, g: CSR) -> tuple[np.ndarray, np.ndarray]:
        urow = np.zeros(g.n + 1, np.uint32)
        ucol = np.zeros(max(2 * g.m, 1), np.uint32)
        self.lib.ref_undirected_csr(*self._args2(g), urow, ucol)
        return urow, ucol[: 2 * g.m]

    def core_decomposition(self, g: CSR) -> tuple[np.ndarray, int]:
        core = np.zeros(max(g.n, 1), np.uint32)
        k = C.c_uint32(0)
        if not self.lib.ref_core_decomposition(*self._args2(g), core, C.byref(k)):
            raise OverflowError("core number does not fit uint32")
        return core[: g.n], int(k.value)

    def core_levels(self, g: CSR) -> tuple[np.ndarray, int, int]:
        core = np.zeros(max(g.n, 1), np.uint32)
        k, r = C.c_uint32(0), C.c_uint32(0)
        if not self.lib.ref_core_levels(*self._args2(g), core, C.byref(k), C.byref(r)):
            raise OverflowError("triangle count >= 2^32")
        return core[: g.n], int(k.value), int(r.value)

    def core_level_density(self, g: CSR, core: np.ndarray, k: int) -> tuple[int, int]:
        a, b = C.c_uint64(0), C.c_uint64(0)
        c = np.ascontiguousarray(core, np.uint32) if g.n else np.zeros(1, np.uint32)
        self.lib.ref_core_level_density(*self._args2(g), c, k, C.byref(a), C.byref(b))
        return int(a.value), int(b.value)


    # ---- densest subgraph (dsg.h) ----
    def _dsg(self, ok, out, setbuf, err, what) -> DsgOut:
        if not ok:
            raise RuntimeError(f"{what}: {err.value.decode()}")
        return DsgOut(int(out[0]), int(out[1]), setbuf[: int(out[5])].copy(), int(out[2]), int(out[3]), int(out[4]))

    def greedy_pp(self, g: CSR, passes: int) -> DsgOut:
        out, setbuf = np.zeros(6, np.uint64), np.zeros(max(g.n, 1), np.uint32)
        per = np.zeros(2 * max(passes, 1), np.uint64)
        err = C.create_string_buffer(256)
        r = self._dsg(self.lib.ref_greedy_pp(*self._args2(g), passes, out, setbuf, per, err, 256), out, setbuf, err,
                      "greedy_pp")
        r.per_pass = [(int(per[2 * i]), int(per[2 * i + 1])) for i in range(passes)]
        return r

    def cpu_greedy_peel(self, g: CSR) -> tuple[int, int]:
        a, b = C.c_uint64(0), C.c_uint64(0)
        if not self.lib.ref_cpu_greedy_peel(*self._args2(g), C.byref(a), C.byref(b)):
            raise RuntimeError("cpu_greedy_peel failed")
        return int(a.value), int(b.value)

    def core_exact(self, g: CSR, core: np.ndarray, use_pruning12: bool = True, seed: "DsgOut | None" = None) -> DsgOut:
        out, setbuf = np.zeros(6, np.uint64), np.zeros(max(g.n, 1), np.uint32)
        err = C.create_string_buffer(256)
        c = np.ascontiguousarray(core, np.uint32) if g.n else np.zeros(1, np.uint32)
        sset = np.ascontiguousarray(seed.set, np.uint32) if seed is not None and len(seed.set) else np.zeros(1, np.uint32)
        slen = len(seed.set) if seed is not None else 0
        ok = self.lib.ref_core_exact(*self._args2(g), c, int(use_pruning12), int(seed is not None), sset, slen,
                                     seed.tri if seed else 0, seed.verts if seed else 0, out, setbuf, err, 256)
        return self._dsg(ok, out, setbuf, err, "core_exact")

    def exact_densest(self, g: CSR) -> DsgOut:
        out, setbuf = np.zeros(6, np.uint64), np.zeros(max(g.n, 1), np.uint32)
        err = C.create_string_buffer(256)
        return self._dsg(self.lib.ref_exact_densest(*self._args2(g), out, setbuf, err, 256), out, setbuf, err,
                         "exact_densest")

    def prune_to_core(self, g: CSR, core: np.ndarray, k: int) -> tuple[CSR, np.ndarray, np.ndarray]:
        rowptr = np.zeros(g.n + 1, np.uint32)
        col, src = np.zeros(max(g.m, 1), np.uint32), np.zeros(max(g.m, 1), np.uint32)
        old, cout = np.zeros(max(g.n, 1), np.uint32), np.zeros(max(g.n, 1), np.uint32)
        c = np.ascontiguousarray(core, np.uint32) if g.n else np.zeros(1, np.uint32)
        n2, m2, mx = C.c_uint32(0), C.c_uint32(0), C.c_uint32(0)
        self.lib.ref_prune_to_core(*self._args2(g), c, k, rowptr, col, src, old, cout, C.byref(n2), C.byref(m2),
                                   C.byref(mx))
        n2, m2 = int(n2.value), int(m2.value)
        return (CSR(n2, m2, rowptr[: n2 + 1].copy(), col[:m2].copy(), src[:m2].copy(), int(mx.value)),
                old[:n2].copy(), cout[:n2].copy())

def _col(g: CSR) -> np.ndarray:
    return g.col if g.m else np.zeros(1, np.uint32)


def _src(g: CSR) -> np.ndarray:
    return g.src if g.m else np.zeros(1, np.uint32)


def _alive(alive: np.ndarray, n: int) -> np.ndarray:
    a = np.ascontiguousarray(alive, dtype=np.uint8)
    return a if n else np.zeros(1, np.uint8)


class RefGraph:
    """The reference's Graph resident in its library: cpu_triangles_omp (graph.h:123) on the whole graph or on a row
    range (the same loop with other bounds)."""

    def __init__(self, ref: Reference, g: CSR):
        self.ref, self.n = ref, g.n
        self.h = ref.lib.ref_graph_new(g.n, g.m, g.rowptr, _col(g), _src(g))

    def triangles_omp(self) -> int:
        return int(self.ref.lib.ref_graph_triangles_omp(self.h))

    def triangles_omp_rows(self, u0: int, u1: int) -> int:
        return int(self.ref.lib.ref_graph_triangles_omp_rows(self.h, u0, u1))

    def triangles_serial_rows(self, u0: int, u1: int) -> int:
        return int(self.ref.lib.ref_graph_triangles_serial_rows(self.h, u0, u1))

    def close(self) -> None:
        if self.h:
            self.ref.lib.ref_graph_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
