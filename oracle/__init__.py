"""CPU oracle for the multi-query traversal path -- TEST INFRASTRUCTURE ONLY.

Loads oracle/liboracle.so (the C restatement in oracle.c of the reference's
cpu_bfs / cpu_sssp / cpu_wcc, puercgp/examples/mtx_loader.hxx:269-356) and,
when it was built here, oracle/_ref/libcgpref.so (those same reference
functions compiled from the reference's own header).  Only the tests,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use this package; the
shipped library never does.
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
        _lib = l
    return _lib


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
