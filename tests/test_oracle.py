"""The CPU oracle pinned against the reference's golden vectors and, when the
reference was compiled here (oracle/_ref), against the reference itself."""
import numpy as np
import pytest

import oracle
from conftest import as_expected, host_csr

INF = 2**31 - 1


def _case(golden, name):
    return next(c for c in golden["cases"] if c["name"] == name)


def test_oracle_bfs_matches_reference_unweighted_mm(golden):
    c = _case(golden, "unweighted_mm")
    g = host_csr(c["graph"])
    for s, exp in zip(c["sources"], c["expect"]):
        assert oracle.bfs(g, s).tolist() == exp


def test_oracle_sssp_matches_reference_weighted_mm(golden):
    c = _case(golden, "weighted_mm")
    g = host_csr(c["graph"])
    for s, exp in zip(c["sources"], c["expect"]):
        np.testing.assert_array_equal(oracle.sssp(g, s), as_expected(exp, np.float32))


@pytest.mark.parametrize("name", ["hybrid_toy", "replenish_toy"])
def test_oracle_known_answers(golden, name):
    c = _case(golden, name)
    g = host_csr(c["graph"])
    for (kind, src), exp in zip(c["queries"], c["expect"]):
        if kind == "bfs":
            assert oracle.bfs(g, src).tolist() == exp
        elif kind == "sssp":
            np.testing.assert_array_equal(oracle.sssp(g, src), as_expected(exp, np.float32))
        else:
            # WCC on a directed toy: the reference GPU push (label = min over
            # vertices that reach v) and weak components agree here ...
            assert oracle.wcc_components(g).tolist() == exp


def test_wcc_directed_semantics_documented(golden):
    # ... while cpu_wcc's in-place sweep follows out-edges only, so on the
    # directed toy it leaves labels at their ids (validate_wcc.cu checks the
    # GPU push result, which is all zeros).
    c = _case(golden, "wcc_toy")
    g = host_csr(c["graph"])
    assert oracle.wcc_components(g).tolist() == c["expect"][0]
    assert oracle.wcc_label_propagation(g).tolist() == [0, 1, 2, 3]


@pytest.mark.parametrize("name", ["rmat8_ref", "grid12_ref"])
def test_oracle_matches_reference_outputs(golden, name):
    c = _case(golden, name)
    g = host_csr(c["graph"])
    for s, b, d in zip(c["sources"], c["bfs"], c["sssp"]):
        assert oracle.bfs(g, s).tolist() == b
        np.testing.assert_array_equal(oracle.sssp(g, s), as_expected(d, np.float32))
    ref_wcc = np.asarray(c["wcc"], np.float32).astype(np.uint32)
    np.testing.assert_array_equal(oracle.wcc_label_propagation(g), ref_wcc)
    np.testing.assert_array_equal(oracle.wcc_components(g), ref_wcc)


def test_oracle_khop_truncates_bfs(golden):
    c = _case(golden, "rmat8_ref")
    g = host_csr(c["graph"])
    s = c["sources"][0]
    full = oracle.bfs(g, s)
    for k in (0, 1, 2, 3):
        kh = oracle.bfs(g, s, max_depth=k)
        exp = np.where(full <= k, full, INF)
        np.testing.assert_array_equal(kh, exp)


def test_oracle_u32_equals_f32_on_integer_weights():
    import cgp_b200 as cgp
    g = cgp.gen_rmat(9, 8, seed=3).with_weights("u32", 1, 64, seed=4)
    gf = cgp.HostCsr(g.row_offsets, g.col_indices, g.weights.astype(np.float32))
    for s in g.pick_sources(4, seed=5):
        du = oracle.sssp(g, int(s))
        df = oracle.sssp(gf, int(s))
        reach = du != 2**32 - 1
        np.testing.assert_array_equal(du[reach].astype(np.float32), df[reach])
        assert np.all(np.isinf(df[~reach]))


def test_oracle_batch_matches_single_queries():
    import cgp_b200 as cgp
    g = cgp.gen_rmat(10, 8, seed=21).with_weights("u32", 1, 64, seed=22)
    src = g.pick_sources(9, seed=23)
    vals, edges = oracle.batch("bfs", g, src, threads=3)
    deg = g.degrees()
    for i, s in enumerate(src):
        d = oracle.bfs(g, int(s))
        np.testing.assert_array_equal(vals[i], d)
        assert edges[i] == int(deg[d != INF].sum())
    svals, _ = oracle.batch("sssp", g, src, threads=2)
    for i, s in enumerate(src):
        np.testing.assert_array_equal(svals[i], oracle.sssp(g, int(s)))


@pytest.mark.skipif(not oracle.has_ref(), reason="reference not compiled here")
def test_oracle_matches_live_reference_on_random_graphs():
    import cgp_b200 as cgp
    for seed in (1, 2):
        g = cgp.gen_rmat(10, 8, seed=seed).with_weights("f32", 0.5, 9.5, seed=seed + 10)
        for s in g.pick_sources(5, seed=seed + 20):
            assert np.array_equal(oracle.bfs(g, int(s)), oracle.ref_bfs(g, int(s)))
            assert np.array_equal(oracle.sssp(g, int(s)), oracle.ref_sssp(g, int(s)))
        np.testing.assert_array_equal(oracle.wcc_components(g),
                                      oracle.ref_wcc(g).astype(np.uint32))


# ------------------------------------------------- generator restatement ---
# The reference arm of the benchmark builds its inputs with oracle/gen.c; it
# must produce the library's arrays exactly, or the two arms would time
# different graphs.
@pytest.mark.parametrize("scale", [6, 12, 16])
def test_oracle_rmat_generator_matches_library(scale):
    import cgp_b200 as cgp
    a = oracle.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed=1)
    b = cgp.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed=1)
    np.testing.assert_array_equal(a.row_offsets, b.row_offsets)
    np.testing.assert_array_equal(a.col_indices, b.col_indices)
    for kind, p0, p1, logn in (("u32", 1, 64, False), ("u32", 1, 255, False),
                               ("f32", 1.0, 100.0, False), ("f32", 0.0, 1.0, True)):
        wa = a.with_weights(kind, p0, p1, seed=2, lognormal=logn).weights
        wb = b.with_weights(kind, p0, p1, seed=2, lognormal=logn).weights
        assert wa.dtype == wb.dtype
        np.testing.assert_array_equal(wa.view(np.uint32), wb.view(np.uint32))
    allowed = (np.arange(a.num_vertices) % 3 == 0).astype(np.uint8)
    np.testing.assert_array_equal(a.pick_sources(100, seed=42), b.pick_sources(100, seed=42))
    np.testing.assert_array_equal(a.pick_sources(50, seed=7, allowed=allowed),
                                  b.pick_sources(50, seed=7, allowed=allowed))


def test_oracle_rmat_unpermuted_and_other_params_match_library():
    import cgp_b200 as cgp
    a = oracle.gen_rmat(10, 8, 0.45, 0.15, 0.15, seed=9, permute=False)
    b = cgp.gen_rmat(10, 8, 0.45, 0.15, 0.15, seed=9, permute=False)
    np.testing.assert_array_equal(a.row_offsets, b.row_offsets)
    np.testing.assert_array_equal(a.col_indices, b.col_indices)


def test_oracle_grid_and_chung_lu_generators_match_library():
    import cgp_b200 as cgp
    for a, b in ((oracle.gen_grid(96, 80, 0.1, 0.001, seed=3), cgp.gen_grid(96, 80, 0.1, 0.001, seed=3)),
                 (oracle.gen_chung_lu(30000, 2.1, 16.0, seed=4),
                  cgp.gen_chung_lu(30000, 2.1, 16.0, seed=4))):
        np.testing.assert_array_equal(a.row_offsets, b.row_offsets)
        np.testing.assert_array_equal(a.col_indices, b.col_indices)
    src = np.array([0, 1, 1, 2, 5, 5, 7], np.int32)
    dst = np.array([1, 0, 2, 2, 6, 6, 0], np.int32)
    a = oracle.csr_from_edges(8, src, dst)
    b = cgp.csr_from_edges(8, src, dst)
    np.testing.assert_array_equal(a.row_offsets, b.row_offsets)
    np.testing.assert_array_equal(a.col_indices, b.col_indices)
