"""Host-side pieces that need no GPU: the C ABI loads and exports every
declared symbol, option defaults, argument validation, generators, loaders."""
import ctypes
from pathlib import Path

import numpy as np
import pytest

import cgp_b200 as cgp
from cgp_b200 import _native as N
from conftest import host_csr

ROOT = Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol():
    lib = cgp.lib()
    declared = cgp.declared_symbols()
    assert len(declared) > 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_library_built_for_sm100a():
    assert b"sm_100a" in cgp.lib().cgp_version()


def test_options_defaults_match_run_options():
    # run_options defaults, puercgp/include/puercgp/core/types.hxx:26-46
    o = N.default_options()
    assert o.traversal_mode == N.MODE_HYBRID
    assert o.pull_frontier_ratio == pytest.approx(0.15)
    assert o.pull_edge_ratio == pytest.approx(0.20)
    assert o.max_iterations == 0 and o.max_queries == 0 and o.discard_results == 0


def test_invalid_arguments_rejected_without_device():
    lib = cgp.lib()
    o = N.default_options()
    q = (N.CgpQuery * 1)()
    out = np.zeros(4, np.int32)
    st = lib.cgp_batch_run(None, q, 1, ctypes.byref(o), out.ctypes.data, 0, 0, None)
    assert st == N.ERR_INVALID_ARG
    assert "graph" in N.last_error()
    h = ctypes.c_void_p()
    row = np.array([0, 1], np.int64)
    col = np.array([0], np.int32)
    st = lib.cgp_graph_create(row.ctypes.data, 3, col.ctypes.data, None, 0, 1, 1, 0,
                              ctypes.byref(h))
    assert st == N.ERR_INVALID_ARG and "offset_bytes" in N.last_error()
    st = lib.cgp_graph_create(row.ctypes.data, 8, col.ctypes.data, None, 7, 1, 1, 0,
                              ctypes.byref(h))
    assert st == N.ERR_INVALID_ARG
    with pytest.raises(ValueError):
        N.check(N.ERR_INVALID_ARG, "x")


def test_query_batch_validation_mirrors_reference():
    # query_batch::validate (core/query_batch.hxx:44-56),
    # hybrid_query_batch::validate (core/query_descriptor.hxx:44-60)
    with pytest.raises(ValueError):
        cgp.QueryBatch([]).validate(0)
    with pytest.raises(ValueError):
        cgp.QueryBatch([1, -2]).validate(0)
    with pytest.raises(ValueError):
        cgp.QueryBatch([1, 2, 3]).validate(2)
    with pytest.raises(ValueError):
        cgp.HybridQueryBatch([]).validate()
    b = cgp.HybridQueryBatch([cgp.QueryDescriptor(0, "bfs"), cgp.QueryDescriptor(1, "sssp"),
                              cgp.QueryDescriptor(0, "wcc")])
    b.validate()
    assert b.bfs_slot_mask() == 0b001 and b.nonbfs_slot_mask() == 0b110
    assert b.has_bfs() and b.has_wcc()
    # no 64-query cap: 200 queries form one valid batch (groups of <= 1024)
    cgp.HybridQueryBatch([cgp.QueryDescriptor(i, "bfs") for i in range(200)]).validate()


def _check_csr_invariants(g):
    row, col = g.row_offsets, g.col_indices
    V = g.num_vertices
    assert row[0] == 0 and row[-1] == len(col)
    assert np.all(np.diff(row) >= 0)
    assert col.min() >= 0 and col.max() < V
    src = np.repeat(np.arange(V), np.diff(row))
    assert not np.any(src == col), "self loop"
    key = src.astype(np.int64) * V + col
    assert np.all(np.diff(key) > 0), "rows not sorted / duplicate entries"
    rkey = col.astype(np.int64) * V + src
    assert np.array_equal(np.sort(rkey), key), "not symmetric"


def test_rmat_generator_invariants_and_determinism():
    a = cgp.gen_rmat(10, 16, seed=1)
    b = cgp.gen_rmat(10, 16, seed=1)
    c = cgp.gen_rmat(10, 16, seed=2)
    assert a.num_vertices == 1024
    _check_csr_invariants(a)
    assert np.array_equal(a.row_offsets, b.row_offsets) and np.array_equal(a.col_indices, b.col_indices)
    assert not np.array_equal(a.col_indices[:100], c.col_indices[:100])
    deg = a.degrees()
    assert deg.max() > 8 * deg.mean()  # skewed degrees
    assert 1.0 * a.num_edges / (2 * 16 * 1024) > 0.5


def test_grid_and_chung_lu_generators():
    g = cgp.gen_grid(40, 30, 0.1, 0.01, seed=3)
    assert g.num_vertices == 1200
    _check_csr_invariants(g)
    assert g.degrees().max() <= 8
    cl = cgp.gen_chung_lu(5000, 2.1, 16.0, seed=4)
    _check_csr_invariants(cl)
    assert cl.degrees().max() > 20 * cl.degrees().mean()


def test_weights_symmetric_and_in_range():
    g = cgp.gen_rmat(9, 8, seed=5).with_weights("u32", 1, 64, seed=6)
    V = g.num_vertices
    src = np.repeat(np.arange(V), g.degrees())
    w = {(int(u), int(v)): int(x) for u, v, x in zip(src, g.col_indices, g.weights)}
    assert all(w[(v, u)] == x for (u, v), x in w.items())
    assert g.weights.dtype == np.uint32 and g.weights.min() >= 1 and g.weights.max() <= 64
    f = cgp.gen_rmat(9, 8, seed=5).with_weights("f32", 0.0, 1.0, seed=7, lognormal=True)
    assert f.weights.dtype == np.float32 and np.all(f.weights > 0)


def test_pick_sources():
    g = cgp.gen_rmat(10, 4, seed=8)
    s = g.pick_sources(50, seed=42)
    assert np.all(g.degrees()[s] >= 1)
    assert np.array_equal(s, g.pick_sources(50, seed=42))
    allowed = np.zeros(g.num_vertices, np.uint8)
    allowed[s[:3]] = 1
    s2 = g.pick_sources(20, seed=1, allowed=allowed)
    assert set(s2.tolist()) <= set(s[:3].tolist())


def test_csr_from_edges():
    g = cgp.csr_from_edges(5, [0, 1, 1, 3, 2], [1, 0, 2, 3, 4], symmetrize=True)
    assert g.row_offsets.tolist() == [0, 1, 3, 5, 5, 6]
    assert g.col_indices.tolist() == [1, 0, 2, 1, 4, 2]


def test_matrix_market_loader_matches_reference_loader(golden, tmp_path):
    for c in golden["cases"]:
        if "mtx" not in c:
            continue
        p = tmp_path / (c["name"] + ".mm")
        p.write_text(c["mtx"])
        g = cgp.load_matrix_market(str(p))
        ref = host_csr(c["graph"])
        assert np.array_equal(g.row_offsets, ref.row_offsets)
        assert np.array_equal(g.col_indices, ref.col_indices)
        assert np.array_equal(g.weights, ref.weights)


def test_matrix_market_symmetric_keeps_duplicates_like_reference(tmp_path):
    p = tmp_path / "s.mm"
    p.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 3\n2 1\n2 1\n3 3\n")
    g = cgp.load_matrix_market(str(p))
    # mirrored off-diagonal entries, the duplicate kept, the self loop kept once
    assert g.row_offsets.tolist() == [0, 2, 4, 5]
    assert g.col_indices.tolist() == [1, 1, 0, 0, 2]


def test_binary_csr_loader(tmp_path):
    np.array([0, 2, 3, 3], np.int32).tofile(tmp_path / "csr_vlist.bin")
    np.array([1, 2, 0], np.int32).tofile(tmp_path / "csr_elist.bin")
    g = cgp.load_binary_csr(str(tmp_path))
    assert g.num_vertices == 3 and g.col_indices.tolist() == [1, 2, 0]
    assert g.weights.tolist() == [1.0, 1.0, 1.0]
    np.array([5, 6, 7], np.int32).tofile(tmp_path / "csr_weightlist.bin")
    assert cgp.load_binary_csr(str(tmp_path)).weights.tolist() == [5.0, 6.0, 7.0]
    np.array([5, 6], np.int32).tofile(tmp_path / "csr_weightlist.bin")
    with pytest.raises(ValueError):
        cgp.load_binary_csr(str(tmp_path))


def _write_gr(path, V, rows_end, dst, edge_bytes=0, data=None, version=1):
    import struct
    with open(path, "wb") as f:
        f.write(struct.pack("<4Q", version, edge_bytes, V, len(dst)))
        f.write(np.asarray(rows_end, np.uint64).tobytes())
        f.write(np.asarray(dst, np.uint32).tobytes())
        if data is not None:
            if len(dst) % 2:
                f.write(b"\0" * 4)
            f.write(np.asarray(data, np.uint32).tobytes())


def test_galois_gr_loader(tmp_path):
    # 5 vertices, 7 edges (odd: the edge data follows 4 bytes of padding)
    rows_end = [2, 3, 3, 6, 7]
    dst = [1, 3, 2, 0, 1, 4, 0]
    data = [5, 6, 7, 8, 9, 10, 11]
    p = tmp_path / "g.gr"
    _write_gr(p, 5, rows_end, dst, 4, data)
    g = cgp.load_galois_gr(str(p))  # the reference reads the topology only
    assert g.row_offsets.tolist() == [0] + rows_end
    assert g.col_indices.tolist() == dst
    assert g.weights is None
    gw = cgp.load_galois_gr(str(p), read_edge_data=True)
    assert gw.weights.dtype == np.uint32 and gw.weights.tolist() == data
    # even edge count: no padding
    p2 = tmp_path / "h.gr"
    _write_gr(p2, 3, [1, 2, 2], [1, 0], 4, [3, 4])
    assert cgp.load_galois_gr(str(p2), read_edge_data=True).weights.tolist() == [3, 4]


def test_galois_gr_loader_rejects_bad_files(tmp_path):
    bad = {
        "version": dict(V=2, rows_end=[1, 1], dst=[1], version=2),
        "range": dict(V=2, rows_end=[1, 1], dst=[5]),
        "ends": dict(V=2, rows_end=[1, 3], dst=[1]),
        "order": dict(V=3, rows_end=[2, 1, 3], dst=[1, 2, 0]),
    }
    for name, kw in bad.items():
        p = tmp_path / f"{name}.gr"
        _write_gr(p, kw["V"], kw["rows_end"], kw["dst"], version=kw.get("version", 1))
        with pytest.raises(ValueError):
            cgp.load_galois_gr(str(p))
    p = tmp_path / "short.gr"
    _write_gr(p, 4, [1, 2, 3, 4], [1, 2, 3, 0])
    p.write_bytes(p.read_bytes()[:-6])
    with pytest.raises(ValueError, match="truncated"):
        cgp.load_galois_gr(str(p))
    with pytest.raises(ValueError):
        cgp.load_galois_gr(str(tmp_path / "missing.gr"))
