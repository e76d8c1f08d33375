"""CPU oracle for the multi-query traversal path -- TEST INFRASTRUCTURE ONLY.

Loads oracle/liboracle.so (the C restatement in oracle.c of the reference's
cpu_bfs / cpu_sssp / cpu_wcc, puercgp/examples/mtx_loader.hxx:269-356) and,
when it was built here, oracle/_ref/libcgpref.so (those same reference
functions compiled from the reference's own header), plus a C restatement
of the library's seeded graph generators (oracle/gen.c) so that the CPU side
of the benchmark builds its inputs without loading the product library.  Only
the tests, __graft_entry__.smoke() and bench.py's CPU legs use this package;
the shipped library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = HERE / "liboracle.so"
_REF = HERE / "_ref" / "libcgpref.so"
_lib = None
_ref = None

KIND_BFS, KIND_SSSP_U32, KIND_SSSP_F32, KIND_KHOP = 0, 1, 2, 3
BFS_INF = 2**31 - 1
U32_INF = 2**32 - 1


def _load():
    global _lib
    if _lib is None:
        if not _LIB.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), str(_LIB)], check=True)
        l = ctypes.CDLL(str(_LIB))
        P = ctypes.c_void_p
        l.oracle_bfs.restype = ctypes.c_int64
        l.oracle_bfs.argtypes = [ctypes.c_int64, P, P, ctypes.c_int32, ctypes.c_int32, P]
        l.oracle_sssp_f32.restype = ctypes.c_int64
        l.oracle_sssp_f32.argtypes = [ctypes.c_int64, P, P, P, ctypes.c_int32, P]
        l.oracle_sssp_u32.restype = ctypes.c_int64
        l.oracle_sssp_u32.argtypes = [ctypes.c_int64, P, P, P, ctypes.c_int32, P]
        l.oracle_wcc_label_propagation.restype = ctypes.c_int32
        l.oracle_wcc_label_propagation.argtypes = [ctypes.c_int64, P, P, ctypes.c_int32, P]
        l.oracle_wcc_components.restype = None
        l.oracle_wcc_components.argtypes = [ctypes.c_int64, P, P, P]
        l.oracle_batch.restype = None
        l.oracle_batch.argtypes = [ctypes.c_int32, ctypes.c_int64, P, P, P, P, P, ctypes.c_int32,
                                   ctypes.c_int32, P, P]
        Csr = ctypes.POINTER(_OracleCsr)
        l.oracle_gen_rmat.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                      ctypes.c_int32, Csr]
        l.oracle_gen_grid.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_uint64, Csr]
        l.oracle_gen_chung_lu.argtypes = [ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_uint64, Csr]
        l.oracle_gen_weights.argtypes = [Csr, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int32, ctypes.c_uint64]
        l.oracle_pick_sources.argtypes = [Csr, ctypes.c_int32, ctypes.c_int32, P,
                                          ctypes.c_uint64, P]
        l.oracle_csr_from_edges.argtypes = [ctypes.c_int64, ctypes.c_int64, P, P, ctypes.c_int32,
                                            Csr]
        l.oracle_csr_free.restype = None
        l.oracle_csr_free.argtypes = [Csr]
        _lib = l
    return _lib


# ------------------------------------------------------------ generators ---
class _OracleCsr(ctypes.Structure):
    _fields_ = [("V", ctypes.c_int64), ("E", ctypes.c_int64),
                ("row", ctypes.POINTER(ctypes.c_int64)), ("col", ctypes.POINTER(ctypes.c_int32)),
                ("w", ctypes.c_void_p), ("weight_kind", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class Graph:
    """Host CSR built by the C generators (int64 offsets, int32 columns,
    optional uint32 / float32 weights)."""

    def __init__(self, row_offsets, col_indices, weights=None):
        self.row_offsets = row_offsets
        self.col_indices = col_indices
        self.weights = weights

    @property
    def num_vertices(self) -> int:
        return len(self.row_offsets) - 1

    @property
    def num_edges(self) -> int:
        return len(self.col_indices)

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_offsets)

    def _c(self):
        c = _OracleCsr()
        row, col = _csr(self)
        self._keep = (row, col)
        c.V, c.E = len(row) - 1, len(col)
        c.row = row.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        c.col = col.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        return c

    def with_weights(self, kind: str, p0: float, p1: float, seed: int = 2,
                     lognormal: bool = False) -> "Graph":
        c = self._c()
        wk = 1 if kind == "u32" else 2
        _check(_load().oracle_gen_weights(ctypes.byref(c), wk, p0, p1, int(lognormal), seed),
               "oracle_gen_weights")
        dt = np.uint32 if wk == 1 else np.float32
        E = self.num_edges
        w = (np.frombuffer((ctypes.c_char * (4 * max(E, 1))).from_address(c.w), dtype=dt)[:E].copy())
        c.row = ctypes.POINTER(ctypes.c_int64)()  # arrays owned by numpy
        c.col = ctypes.POINTER(ctypes.c_int32)()
        _load().oracle_csr_free(ctypes.byref(c))
        return Graph(self.row_offsets, self.col_indices, w)

    def pick_sources(self, count: int, seed: int = 42, min_degree: int = 1,
                     allowed=None) -> np.ndarray:
        c = self._c()
        out = np.zeros(count, np.int32)
        al = None
        if allowed is not None:
            allowed = np.ascontiguousarray(allowed, np.uint8)
            al = allowed.ctypes.data
        _check(_load().oracle_pick_sources(ctypes.byref(c), count, min_degree, al, seed,
                                           out.ctypes.data), "oracle_pick_sources")
        return out


def _check(rc: int, what: str):
    if rc != 0:
        raise (MemoryError if rc == 2 else ValueError)(f"{what} failed ({rc})")


def _take(c: _OracleCsr) -> Graph:
    V, E = c.V, c.E
    row = np.ctypeslib.as_array(c.row, shape=(V + 1,)).copy()
    col = np.ctypeslib.as_array(c.col, shape=(max(E, 1),))[:E].copy()
    _load().oracle_csr_free(ctypes.byref(c))
    return Graph(row, col)


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, seed: int = 1, permute: bool = True) -> Graph:
    h = _OracleCsr()
    _check(_load().oracle_gen_rmat(scale, edge_factor, a, b, c, seed, int(permute),
                                   ctypes.byref(h)), "oracle_gen_rmat")
    return _take(h)


def gen_grid(rows: int, cols: int, delete_frac: float = 0.1, shortcut_frac: float = 0.001,
             seed: int = 1) -> Graph:
    h = _OracleCsr()
    _check(_load().oracle_gen_grid(rows, cols, delete_frac, shortcut_frac, seed,
                                   ctypes.byref(h)), "oracle_gen_grid")
    return _take(h)


def gen_chung_lu(num_vertices: int, exponent: float = 2.1, mean_degree: float = 16.0,
                 seed: int = 1) -> Graph:
    h = _OracleCsr()
    _check(_load().oracle_gen_chung_lu(num_vertices, exponent, mean_degree, seed,
                                       ctypes.byref(h)), "oracle_gen_chung_lu")
    return _take(h)


def csr_from_edges(num_vertices: int, src, dst, symmetrize: bool = True) -> Graph:
    s = np.ascontiguousarray(src, np.int32)
    d = np.ascontiguousarray(dst, np.int32)
    h = _OracleCsr()
    _check(_load().oracle_csr_from_edges(num_vertices, len(s), s.ctypes.data, d.ctypes.data,
                                         int(symmetrize), ctypes.byref(h)),
           "oracle_csr_from_edges")
    return _take(h)


def _csr(g):
    row = np.ascontiguousarray(g.row_offsets, np.int64)
    col = np.ascontiguousarray(g.col_indices, np.int32)
    return row, col


def bfs(g, source: int, max_depth: int = -1) -> np.ndarray:
    """FIFO BFS depths (int32, INT32_MAX unreached); max_depth >= 0: k-hop."""
    row, col = _csr(g)
    out = np.empty(len(row) - 1, np.int32)
    _load().oracle_bfs(len(row) - 1, row.ctypes.data, col.ctypes.data, source, max_depth,
                       out.ctypes.data)
    return out


def sssp(g, source: int, weights=None) -> np.ndarray:
    """Dijkstra: float32 (left-fold fp32 sums) for float weights, exact uint32
    for integer or absent weights."""
    row, col = _csr(g)
    w = g.weights if weights is None else weights
    V = len(row) - 1
    if w is not None and np.asarray(w).dtype == np.float32:
        w = np.ascontiguousarray(w, np.float32)
        out = np.empty(V, np.float32)
        _load().oracle_sssp_f32(V, row.ctypes.data, col.ctypes.data, w.ctypes.data, source,
                                out.ctypes.data)
    else:
        wp = None
        if w is not None:
            w = np.ascontiguousarray(w, np.uint32)
            wp = w.ctypes.data
        out = np.empty(V, np.uint32)
        _load().oracle_sssp_u32(V, row.ctypes.data, col.ctypes.data, wp, source, out.ctypes.data)
    return out


def wcc_label_propagation(g, max_sweeps: int = 10000) -> np.ndarray:
    """cpu_wcc restated: in-place min-label sweeps along CSR rows (uint32)."""
    row, col = _csr(g)
    out = np.empty(len(row) - 1, np.uint32)
    _load().oracle_wcc_label_propagation(len(row) - 1, row.ctypes.data, col.ctypes.data,
                                         max_sweeps, out.ctypes.data)
    return out


def wcc_components(g) -> np.ndarray:
    """Minimum vertex id of each weak component (uint32)."""
    row, col = _csr(g)
    out = np.empty(len(row) - 1, np.uint32)
    _load().oracle_wcc_components(len(row) - 1, row.ctypes.data, col.ctypes.data, out.ctypes.data)
    return out


def batch(kind: str, g, sources, khop=None, threads: int | None = None):
    """Runs independent queries over host threads.  Returns (values[q][v],
    edges[q]) where edges[q] = sum of out-degrees of vertices reached by q."""
    row, col = _csr(g)
    V = len(row) - 1
    src = np.ascontiguousarray(sources, np.int32)
    nq = len(src)
    w = g.weights
    if kind == "bfs":
        k, dt, wp = KIND_BFS, np.int32, None
    elif kind == "khop":
        k, dt, wp = KIND_KHOP, np.int32, None
    elif w is not None and np.asarray(w).dtype == np.float32:
        w = np.ascontiguousarray(w, np.float32)
        k, dt, wp = KIND_SSSP_F32, np.float32, w.ctypes.data
    else:
        if w is not None:
            w = np.ascontiguousarray(w, np.uint32)
        k, dt, wp = KIND_SSSP_U32, np.uint32, (None if w is None else w.ctypes.data)
    kh = None
    if khop is not None:
        kh = np.ascontiguousarray(khop, np.int32)
    out = np.empty((nq, V), dt)
    edges = np.zeros(nq, np.int64)
    _load().oracle_batch(k, V, row.ctypes.data, col.ctypes.data, wp, src.ctypes.data,
                         None if kh is None else kh.ctypes.data, nq,
                         threads or os.cpu_count() or 1, out.ctypes.data, edges.ctypes.data)
    return out, edges


# ------------------------------------------------------------ reference ---
def has_ref() -> bool:
    return _REF.exists()


def _ref_lib():
    global _ref
    if _ref is None:
        l = ctypes.CDLL(str(_REF))
        P = ctypes.c_void_p
        for name, args in {
            "ref_cpu_bfs": [ctypes.c_int64, P, P, ctypes.c_int32, P],
            "ref_cpu_sssp": [ctypes.c_int64, P, P, P, ctypes.c_int32, P],
            "ref_cpu_wcc": [ctypes.c_int64, P, P, ctypes.c_int32, P],
            "ref_load_matrix_market": [ctypes.c_char_p, P, P, P, P, P],
            "ref_batch": [ctypes.c_int32, ctypes.c_int64, P, P, P, P, ctypes.c_int32,
                          ctypes.c_int32, P],
        }.items():
            getattr(l, name).restype = ctypes.c_int
            getattr(l, name).argtypes = args
        _ref = l
    return _ref


def ref_bfs(g, source: int) -> np.ndarray:
    row, col = _csr(g)
    out = np.empty(len(row) - 1, np.int32)
    _ref_lib().ref_cpu_bfs(len(row) - 1, row.ctypes.data, col.ctypes.data, source,
                           out.ctypes.data)
    return out


def ref_sssp(g, source: int) -> np.ndarray:
    row, col = _csr(g)
    w = None if g.weights is None else np.ascontiguousarray(g.weights, np.float32)
    out = np.empty(len(row) - 1, np.float32)
    _ref_lib().ref_cpu_sssp(len(row) - 1, row.ctypes.data, col.ctypes.data,
                            None if w is None else w.ctypes.data, source, out.ctypes.data)
    return out


def ref_wcc(g, max_iterations: int = 10000) -> np.ndarray:
    row, col = _csr(g)
    out = np.empty(len(row) - 1, np.float32)
    _ref_lib().ref_cpu_wcc(len(row) - 1, row.ctypes.data, col.ctypes.data, max_iterations,
                           out.ctypes.data)
    return out


def ref_load_matrix_market(path: str):
    V, E = ctypes.c_int64(), ctypes.c_int64()
    l = _ref_lib()
    if l.ref_load_matrix_market(str(path).encode(), ctypes.byref(V), ctypes.byref(E), None, None,
                                None) != 0:
        raise ValueError(f"reference loader rejected {path}")
    row = np.empty(V.value + 1, np.int64)
    col = np.empty(max(E.value, 1), np.int32)
    w = np.empty(max(E.value, 1), np.float32)
    l.ref_load_matrix_market(str(path).encode(), ctypes.byref(V), ctypes.byref(E), row.ctypes.data,
                             col.ctypes.data, w.ctypes.data)
    return row, col[:E.value], w[:E.value]


def ref_batch(kind: str, g, sources, threads: int | None = None) -> np.ndarray:
    """The reference's cpu_bfs (kind 'bfs') or cpu_sssp (kind 'sssp') over
    host threads; query-major int32 / float32."""
    row, col = _csr(g)
    V = len(row) - 1
    src = np.ascontiguousarray(sources, np.int32)
    w = None if g.weights is None else np.ascontiguousarray(g.weights, np.float32)
    out = np.empty((len(src), V), np.int32 if kind == "bfs" else np.float32)
    _ref_lib().ref_batch(0 if kind == "bfs" else 2, V, row.ctypes.data, col.ctypes.data,
                         None if w is None else w.ctypes.data, src.ctypes.data, len(src),
                         threads or os.cpu_count() or 1, out.ctypes.data)
    return out
