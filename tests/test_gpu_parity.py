"""Parity of the CUDA path with the CPU oracle, through the C ABI.

Bit-exact everywhere: int32 BFS / k-hop depths, uint32 or float32 SSSP
distances (compared with ==), uint32 WCC labels.
"""
import numpy as np
import pytest

import cgp_b200 as cgp
import oracle
from conftest import as_expected, host_csr

pytestmark = pytest.mark.gpu
INF = 2**31 - 1


@pytest.fixture(scope="module")
def rmat_u32():
    g = cgp.gen_rmat(12, 8, seed=101).with_weights("u32", 1, 64, seed=102)
    return g, cgp.CsrGraph(g)


@pytest.fixture(scope="module")
def rmat_f32():
    g = cgp.gen_rmat(11, 8, seed=103).with_weights("f32", 1.0, 100.0, seed=104)
    return g, cgp.CsrGraph(g)


@pytest.fixture(scope="module")
def grid_f32():
    g = cgp.gen_grid(40, 50, 0.1, 0.01, seed=105).with_weights("f32", 1.0, 100.0, seed=106)
    return g, cgp.CsrGraph(g)


def _bfs(descs_src, graph, opts, layout="query"):
    r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "bfs") for s in descs_src], opts,
                      layout=layout)
    return r


@pytest.mark.parametrize("nq", [1, 5, 64, 65, 130, 256])
@pytest.mark.parametrize("mode", ["push", "pull", "hybrid"])
def test_bfs_parity(rmat_u32, nq, mode):
    g, graph = rmat_u32
    src = g.pick_sources(nq, seed=nq)
    ref, _ = oracle.batch("bfs", g, src)
    r = _bfs(src, graph, cgp.RunOptions(traversal_mode=mode))
    assert r.values.dtype == np.int32
    np.testing.assert_array_equal(r.values, ref)
    if mode == "push":
        assert r.pull_levels == 0
    if mode == "pull":
        assert r.push_levels == 0


@pytest.mark.parametrize("depth", ["planes", "direct"])
@pytest.mark.parametrize("layout", ["vertex", "query"])
def test_bfs_depth_modes_and_layouts(rmat_u32, depth, layout):
    g, graph = rmat_u32
    src = g.pick_sources(100, seed=7)
    ref, _ = oracle.batch("bfs", g, src)
    r = _bfs(src, graph, cgp.RunOptions(depth_mode=depth), layout=layout)
    got = r.values if layout == "query" else r.values.T
    np.testing.assert_array_equal(got, ref)
    assert r.depth_mode == depth


@pytest.mark.parametrize("opts", [
    dict(use_cuda_graph=False), dict(levels_per_sync=1), dict(levels_per_sync=3),
    dict(heavy_degree=16), dict(heavy_degree=64, traversal_mode="pull"),
    dict(mask_words=16), dict(pull_edge_ratio=0.0, pull_frontier_ratio=0.0),
])
def test_bfs_execution_knobs_do_not_change_results(rmat_u32, opts):
    g, graph = rmat_u32
    src = g.pick_sources(70, seed=3)
    ref, _ = oracle.batch("bfs", g, src)
    r = _bfs(src, graph, cgp.RunOptions(**opts))
    np.testing.assert_array_equal(r.values, ref)


def test_bfs_multiple_groups(rmat_u32):
    g, graph = rmat_u32
    src = g.pick_sources(1100, seed=9)
    ref, _ = oracle.batch("bfs", g, src)
    r = _bfs(src, graph, cgp.RunOptions())
    assert r.groups == 2
    np.testing.assert_array_equal(r.values, ref)


def test_bfs_int64_offsets():
    g = cgp.gen_rmat(11, 8, seed=33)
    graph = cgp.CsrGraph(g, offsets64=True)
    src = g.pick_sources(40, seed=4)
    ref, _ = oracle.batch("bfs", g, src)
    np.testing.assert_array_equal(_bfs(src, graph, cgp.RunOptions()).values, ref)


def test_bfs_deep_graph_grows_depth_planes():
    n = 700  # depth 699 needs 10 depth planes; the engine starts with 8
    g = cgp.csr_from_edges(n, list(range(n - 1)), list(range(1, n)))
    graph = cgp.CsrGraph(g)
    src = [0, 350, 699] * 6
    ref, _ = oracle.batch("bfs", g, src)
    r = _bfs(src, graph, cgp.RunOptions(depth_mode="planes"))
    np.testing.assert_array_equal(r.values, ref)
    assert r.iterations >= 699


def test_bfs_directed_graph_pull_uses_transpose():
    rng = np.random.default_rng(5)
    V = 3000
    s = rng.integers(0, V, 20000)
    d = rng.integers(0, V, 20000)
    g = cgp.csr_from_edges(V, s, d, symmetrize=False)
    graph = cgp.CsrGraph(g)
    assert not graph.symmetric
    src = g.pick_sources(50, seed=6)
    ref, _ = oracle.batch("bfs", g, src)
    for mode in ("push", "pull", "hybrid"):
        np.testing.assert_array_equal(_bfs(src, graph, cgp.RunOptions(traversal_mode=mode)).values, ref)


@pytest.mark.parametrize("nq", [1, 33, 64, 200])
def test_sssp_u32_parity(rmat_u32, nq):
    g, graph = rmat_u32
    src = g.pick_sources(nq, seed=50 + nq)
    ref, _ = oracle.batch("sssp", g, src)
    r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src], layout="query")
    assert r.values.dtype == np.uint32
    np.testing.assert_array_equal(r.values, ref)


@pytest.mark.parametrize("which", ["rmat", "grid"])
def test_sssp_f32_parity(rmat_f32, grid_f32, which):
    g, graph = rmat_f32 if which == "rmat" else grid_f32
    src = g.pick_sources(80, seed=12)
    ref, _ = oracle.batch("sssp", g, src)
    r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src], layout="query")
    assert r.values.dtype == np.float32
    np.testing.assert_array_equal(r.values, ref)  # exact: least fixpoint of fp32 left folds


def test_sssp_heavy_paths(rmat_u32):
    g, graph = rmat_u32
    src = g.pick_sources(90, seed=77)
    ref, _ = oracle.batch("sssp", g, src)
    r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src],
                      cgp.RunOptions(heavy_degree=8), layout="query")
    np.testing.assert_array_equal(r.values, ref)


def test_wcc_parity(rmat_u32, grid_f32):
    for g, graph in (rmat_u32, grid_f32):
        r = cgp.run("wcc", graph, [0])
        np.testing.assert_array_equal(r.values[:, 0], oracle.wcc_components(g))
        np.testing.assert_array_equal(r.values[:, 0], oracle.wcc_label_propagation(g))


def test_wcc_labels_stable_over_repeated_runs(rmat_u32, grid_f32):
    # the label pass runs concurrently with nothing that may rewrite a
    # finished label; repeated runs catch a late path-shortening store
    for g, graph in (rmat_u32, grid_f32):
        want = oracle.wcc_components(g)
        for _ in range(40):
            np.testing.assert_array_equal(cgp.run("wcc", graph, [0]).values[:, 0], want)


def test_khop_parity(rmat_u32):
    g, graph = rmat_u32
    src = g.pick_sources(60, seed=14)
    ks = [2 + (i % 5) for i in range(60)]
    ref, _ = oracle.batch("khop", g, src, khop=ks)
    r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "khop", k) for s, k in zip(src, ks)],
                      layout="query")
    np.testing.assert_array_equal(r.values, ref)


@pytest.mark.parametrize("mode", ["push", "hybrid"])
def test_mixed_batch_parity(rmat_u32, mode):
    g, graph = rmat_u32
    src = g.pick_sources(150, seed=15)
    kinds = ["bfs", "sssp", "khop", "wcc", "bfs", "sssp"]
    descs = [cgp.QueryDescriptor(int(s), kinds[i % 6], 3) for i, s in enumerate(src)]
    r = cgp.run_heterogeneous(graph, cgp.HybridQueryBatch(descs),
                              options=cgp.RunOptions(traversal_mode=mode), layout="query")
    wcc = oracle.wcc_components(g)
    for i, d in enumerate(descs):
        if d.kind == "bfs":
            np.testing.assert_array_equal(r.values[i].view(np.int32), oracle.bfs(g, d.source))
        elif d.kind == "khop":
            np.testing.assert_array_equal(r.values[i].view(np.int32), oracle.bfs(g, d.source, 3))
        elif d.kind == "sssp":
            np.testing.assert_array_equal(r.values[i], oracle.sssp(g, d.source))
        else:
            np.testing.assert_array_equal(r.values[i], wcc)


def test_device_output_buffer(rmat_u32):
    import torch
    g, graph = rmat_u32
    src = g.pick_sources(64, seed=16)
    ref, _ = oracle.batch("bfs", g, src)
    out = torch.empty((g.num_vertices, 64), dtype=torch.int32, device="cuda")
    cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "bfs") for s in src], out=out)
    np.testing.assert_array_equal(out.cpu().numpy().T, ref)


def test_repeat_runs_are_deterministic(rmat_u32):
    g, graph = rmat_u32
    src = g.pick_sources(64, seed=17)
    a = _bfs(src, graph, cgp.RunOptions()).values
    b = _bfs(src, graph, cgp.RunOptions()).values
    assert np.array_equal(a, b)


# ------------------------------------------------ reference known answers
def _case(golden, name):
    return next(c for c in golden["cases"] if c["name"] == name)


def _typed(kind, vec, graph):
    """Expected 4-byte words: SSSP is float32 on float-weighted graphs and
    uint32 (UINT32_MAX unreached) otherwise; BFS int32; WCC uint32."""
    if kind == "sssp":
        f = as_expected(vec, np.float32)
        if graph.weight_kind == 2:
            return f.view(np.uint32)
        out = np.full(len(f), 2**32 - 1, np.uint32)
        fin = np.isfinite(f)
        out[fin] = f[fin].astype(np.uint32)
        return out
    return np.asarray(vec, np.int64).astype(np.uint32)


@pytest.mark.parametrize("name", ["hybrid_toy", "replenish_toy", "wcc_toy"])
def test_reference_known_answers(golden, name):
    c = _case(golden, name)
    g = host_csr(c["graph"])
    graph = cgp.CsrGraph(g)
    descs = [cgp.QueryDescriptor(s, k) for k, s in c["queries"]]
    r = cgp.run_batch(graph, descs, cgp.RunOptions(traversal_mode="push"), layout="query")
    for i, ((k, _), exp) in enumerate(zip(c["queries"], c["expect"])):
        np.testing.assert_array_equal(r.values[i], _typed(k, exp, graph))


def test_reference_mm_fixtures(golden):
    for name in ("unweighted_mm", "weighted_mm"):
        c = _case(golden, name)
        g = host_csr(c["graph"])
        graph = cgp.CsrGraph(g)
        kind = c["kind"]
        r = cgp.run(kind, graph, c["sources"])
        for i, exp in enumerate(c["expect"]):
            got = r.values[:, i]
            if kind == "bfs":
                assert got.tolist() == exp
            else:
                np.testing.assert_array_equal(got, as_expected(exp, np.float32))


@pytest.mark.parametrize("name", ["rmat8_ref", "grid12_ref"])
def test_reference_outputs_on_seeded_graphs(golden, name):
    c = _case(golden, name)
    g = host_csr(c["graph"])
    graph = cgp.CsrGraph(g)
    rb = cgp.run("bfs", graph, c["sources"])
    rs = cgp.run("sssp", graph, c["sources"])
    for i in range(len(c["sources"])):
        assert rb.values[:, i].tolist() == c["bfs"][i]
        np.testing.assert_array_equal(rs.values[:, i], as_expected(c["sssp"][i], np.float32))
    rw = cgp.run("wcc", graph, [0])
    np.testing.assert_array_equal(rw.values[:, 0], np.asarray(c["wcc"], np.float32).astype(np.uint32))


def test_one_push_level_like_smoke_hybrid_push(golden):
    c = _case(golden, "push_one_level")
    g = host_csr(c["graph"])
    graph = cgp.CsrGraph(g)
    descs = [cgp.QueryDescriptor(s, k) for k, s in c["queries"]]
    e = cgp.Enactor(graph, descs, cgp.RunOptions(traversal_mode="push", depth_mode="direct"))
    e.prepare_frontier()
    n = e.loop("push")
    vs, ms = e.frontier()
    assert n == 2 and sorted(vs.tolist()) == c["expect_next_frontier"]["vertices"]
    assert all(int(m[0]) == c["expect_next_frontier"]["mask"] for m in ms)
    vals = e.values("query")
    for i, ((k, _), exp) in enumerate(zip(c["queries"], c["expect"])):
        np.testing.assert_array_equal(vals[i], _typed(k, exp, graph))
    assert not e.is_converged()
    while not e.is_converged():
        e.loop("hybrid")
    e.close()


def test_prepare_frontier_like_smoke_hybrid_init(golden):
    c = _case(golden, "hybrid_init")
    g = host_csr(c["graph"])
    graph = cgp.CsrGraph(g)
    descs = [cgp.QueryDescriptor(s, k) for k, s in c["queries"]]
    e = cgp.Enactor(graph, descs, cgp.RunOptions(depth_mode="direct"))
    e.prepare_frontier()
    vs, ms = e.frontier()
    got = {str(int(v)): int(m[0]) for v, m in zip(vs, ms)}
    assert got == c["expect_frontier"]
    vals = e.values("query")
    for i, ((k, _), exp) in enumerate(zip(c["queries"], c["expect"])):
        np.testing.assert_array_equal(vals[i], _typed(k, exp, graph))


def test_convergence_masks_like_smoke_replenish(golden):
    c = _case(golden, "convergence_levels")
    g = host_csr(c["graph"])
    graph = cgp.CsrGraph(g)
    descs = [cgp.QueryDescriptor(s, k) for k, s in c["queries"]]
    r = cgp.run_batch(graph, descs, cgp.RunOptions(traversal_mode="push", profile_iterations=True))
    assert r.iterations == c["expect_iterations"]
    masks = [p.query_convergence_mask for p in r.iteration_profiles]
    assert masks == c["expect_masks"]
    for a, b in zip(masks, masks[1:]):
        assert b & ~a == 0  # monotone


def test_enactor_steps_equal_enact(rmat_u32):
    g, graph = rmat_u32
    src = g.pick_sources(100, seed=19)
    descs = [cgp.QueryDescriptor(int(s), "bfs") for s in src]
    e = cgp.Enactor(graph, descs)
    e.prepare_frontier()
    steps = 0
    while not e.is_converged():
        e.loop("pull" if steps % 2 else "push")
        steps += 1
    ref, _ = oracle.batch("bfs", g, src)
    np.testing.assert_array_equal(e.values("query").view(np.int32), ref)
    e.prepare_frontier()
    e.enact()
    np.testing.assert_array_equal(e.values("query").view(np.int32), ref)


def test_invalid_batches_raise(rmat_u32):
    g, graph = rmat_u32
    with pytest.raises(ValueError):
        cgp.run("bfs", graph, [])
    with pytest.raises(ValueError):
        cgp.run("bfs", graph, [g.num_vertices])
    with pytest.raises(ValueError):
        cgp.run("bfs", graph, [1, 2, 3], options=cgp.RunOptions(max_queries=2))


def test_autotune_keeps_results_and_caches(rmat_u32):
    import time
    g, graph = rmat_u32
    src = g.pick_sources(160, seed=21)
    descs = [cgp.QueryDescriptor(int(s), "bfs" if i % 2 else "sssp") for i, s in enumerate(src)]
    t0 = time.perf_counter()
    opts = cgp.autotune(graph, descs, reps=1)
    t1 = time.perf_counter()
    again = cgp.autotune(graph, descs, reps=1)
    t2 = time.perf_counter()
    assert again == opts and (t2 - t1) < (t1 - t0)
    assert opts.mask_words in (0, 1, 2, 4) and opts.heavy_degree >= 0
    r = cgp.run_batch(graph, descs, opts, layout="query")
    for i, d in enumerate(descs):
        exp = oracle.bfs(g, d.source).view(np.uint32) if d.kind == "bfs" else oracle.sssp(g, d.source)
        np.testing.assert_array_equal(r.values[i], exp)


@pytest.mark.parametrize("opts", [dict(dense_unroll=2), dict(dense_unroll=1, heavy_degree=64),
                                  dict(dense_unroll=2, heavy_degree=16, mask_words=8)])
def test_sssp_execution_knobs_do_not_change_results(rmat_u32, opts):
    g, graph = rmat_u32
    src = g.pick_sources(300, seed=23)
    ref, _ = oracle.batch("sssp", g, src)
    r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src],
                      cgp.RunOptions(**opts), layout="query")
    np.testing.assert_array_equal(r.values, ref)


# ------------------------------------------------------------- SSSP gather
# Dense SSSP levels gather over in-edges (pull CSR + reverse-edge weights).
@pytest.mark.parametrize("opts", [
    dict(traversal_mode="pull"),
    dict(traversal_mode="hybrid", sssp_pull_edge_ratio=0.02, sssp_pull_pair_ratio=0.0),
    dict(traversal_mode="hybrid", sssp_pull_edge_ratio=0.0),
    dict(traversal_mode="pull", heavy_degree=16),
    dict(traversal_mode="hybrid", sssp_pull_edge_ratio=0.05, sssp_pull_pair_ratio=0.0, heavy_degree=32, mask_words=16),
])
@pytest.mark.parametrize("nq", [62, 70, 72])  # vector rows (uint2 / uint4) and scalar rows
def test_sssp_gather_parity(rmat_u32, rmat_f32, grid_f32, opts, nq):
    for g, graph in (rmat_u32, rmat_f32, grid_f32):
        src = g.pick_sources(nq, seed=31)
        ref, _ = oracle.batch("sssp", g, src)
        r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src],
                          cgp.RunOptions(profile_iterations=True, **opts), layout="query")
        np.testing.assert_array_equal(r.values, ref)
        for p in r.iteration_profiles:  # work counters are per vertex / per edge
            assert p.sssp_pull_vertices <= g.num_vertices
            assert p.sssp_pull_edges <= g.num_edges
        modes = {p.sssp_mode for p in r.iteration_profiles}
        if opts.get("sssp_pull_edge_ratio", 1) == 0.0:
            assert modes == {"push"}
        else:
            assert "pull" in modes


def _weighted_variant(g, w, kind):
    return cgp.HostCsr(g.row_offsets, g.col_indices,
                       np.ascontiguousarray(w, np.uint32 if kind == "u32" else np.float32))


@pytest.mark.parametrize("kind", ["u32", "f32"])
def test_sssp_gather_uses_reverse_edge_weights(kind):
    """Symmetric structure, asymmetric weights: a gather must relax u -> v
    with w(u, v), the weight stored in u's list, not v's."""
    rng = np.random.default_rng(41)
    base = cgp.gen_rmat(11, 8, seed=42)
    w = (rng.integers(1, 100, base.num_edges) if kind == "u32"
         else rng.uniform(0.5, 50.0, base.num_edges))
    g = _weighted_variant(base, w, kind)
    graph = cgp.CsrGraph(g)
    assert graph.symmetric
    src = g.pick_sources(40, seed=43)
    ref, _ = oracle.batch("sssp", g, src)
    for mode in ("push", "pull", "hybrid"):
        r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src],
                          cgp.RunOptions(traversal_mode=mode, sssp_pull_edge_ratio=0.01, sssp_pull_pair_ratio=0.0),
                          layout="query")
        np.testing.assert_array_equal(r.values, ref)


def test_sssp_gather_unsorted_lists_and_directed():
    """Unsorted adjacency lists (the transpose is stored) and a directed
    weighted graph (gather over the transposed CSR and weights)."""
    rng = np.random.default_rng(44)
    base = cgp.gen_rmat(11, 8, seed=45)
    row, col = base.row_offsets, base.col_indices.copy()
    for v in range(base.num_vertices):  # shuffle every list in place
        a, b = row[v], row[v + 1]
        col[a:b] = rng.permutation(col[a:b])
    w = rng.integers(1, 64, base.num_edges)
    g1 = cgp.HostCsr(row, col, np.ascontiguousarray(w, np.uint32))
    V = 2500
    s = rng.integers(0, V, 30000)
    d = rng.integers(0, V, 30000)
    dg = cgp.csr_from_edges(V, s, d, symmetrize=False)
    g2 = cgp.HostCsr(dg.row_offsets, dg.col_indices,
                     np.ascontiguousarray(rng.uniform(1.0, 10.0, dg.num_edges), np.float32))
    for g in (g1, g2):
        graph = cgp.CsrGraph(g)
        src = g.pick_sources(50, seed=46)
        ref, _ = oracle.batch("sssp", g, src)
        for mode in ("pull", "hybrid"):
            r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src],
                              cgp.RunOptions(traversal_mode=mode, sssp_pull_edge_ratio=0.01, sssp_pull_pair_ratio=0.0,
                                             heavy_degree=24), layout="query")
            np.testing.assert_array_equal(r.values, ref)


@pytest.mark.parametrize("ratio", [0.01, 0.5])
def test_mixed_batch_with_sssp_gather(rmat_u32, ratio):
    g, graph = rmat_u32
    src = g.pick_sources(150, seed=47)
    kinds = ["bfs", "sssp", "khop", "sssp"]
    descs = [cgp.QueryDescriptor(int(s), kinds[i % 4], 2) for i, s in enumerate(src)]
    r = cgp.run_heterogeneous(graph, cgp.HybridQueryBatch(descs),
                              options=cgp.RunOptions(sssp_pull_edge_ratio=ratio, sssp_pull_pair_ratio=0.0), layout="query")
    for i, d in enumerate(descs):
        if d.kind == "bfs":
            np.testing.assert_array_equal(r.values[i].view(np.int32), oracle.bfs(g, d.source))
        elif d.kind == "khop":
            np.testing.assert_array_equal(r.values[i].view(np.int32), oracle.bfs(g, d.source, 2))
        else:
            np.testing.assert_array_equal(r.values[i], oracle.sssp(g, d.source))


@pytest.mark.parametrize("layout", ["vertex", "query"])
@pytest.mark.parametrize("order", ["blocks", "interleaved", "with_wcc"])
def test_large_mixed_batch_split_by_kind(rmat_u32, layout, order):
    """>= 64 BFS and >= 64 SSSP queries run as separate per-kind groups; the
    host result blocks are copied while later groups traverse (contiguous
    blocks) or in one copy at the end (interleaved kinds, WCC columns)."""
    g, graph = rmat_u32
    src = g.pick_sources(180, seed=48)
    if order == "interleaved":
        kinds = ["bfs" if i % 2 else "sssp" for i in range(180)]
    else:
        kinds = ["bfs"] * 100 + ["sssp"] * 80
    descs = [cgp.QueryDescriptor(int(s), k) for s, k in zip(src, kinds)]
    if order == "with_wcc":
        descs.append(cgp.QueryDescriptor(0, "wcc"))
    r = cgp.run_heterogeneous(graph, cgp.HybridQueryBatch(descs), layout=layout)
    assert r.groups == 2
    vals = r.values if layout == "query" else r.values.T
    for i, d in enumerate(descs):
        if d.kind == "bfs":
            np.testing.assert_array_equal(vals[i].view(np.int32), oracle.bfs(g, d.source))
        elif d.kind == "sssp":
            np.testing.assert_array_equal(vals[i], oracle.sssp(g, d.source))
        else:
            np.testing.assert_array_equal(vals[i], oracle.wcc_components(g))


@pytest.mark.parametrize("wrange", [(1, 64), (500, 4000), (1 << 20, 1 << 21), (1 << 30, 3 << 30)])
@pytest.mark.parametrize("opts", [dict(traversal_mode="pull"),
                                  dict(sssp_pull_edge_ratio=0.05, sssp_pull_pair_ratio=0.0, heavy_degree=32)])
def test_sssp_gather_weight_ranges(wrange, opts):
    """256-slot gathers and scatters with small, medium, large and near-overflow
    integer weights (sums saturate at UINT32_MAX exactly like the oracle's)."""
    g = cgp.gen_rmat(12, 8, seed=121).with_weights("u32", wrange[0], wrange[1], seed=122)
    graph = cgp.CsrGraph(g)
    src = g.pick_sources(256, seed=123)
    ref, _ = oracle.batch("sssp", g, src)
    r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src],
                      cgp.RunOptions(mask_words=4, **opts), layout="query")
    assert r.mask_words == 4
    np.testing.assert_array_equal(r.values, ref)


def test_sssp_gather_mixed_group(rmat_u32):
    """A 256-slot group with 32 BFS slots: the gathers read whole rows, BFS
    depths included, and must update only the SSSP slots."""
    g, graph = rmat_u32
    src = g.pick_sources(256, seed=124)
    descs = [cgp.QueryDescriptor(int(s), "bfs" if i % 8 == 0 else "sssp")
             for i, s in enumerate(src)]
    r = cgp.run_heterogeneous(graph, cgp.HybridQueryBatch(descs),
                              options=cgp.RunOptions(traversal_mode="pull", mask_words=4),
                              layout="query")
    assert r.groups == 1
    for i, d in enumerate(descs):
        if d.kind == "bfs":
            np.testing.assert_array_equal(r.values[i].view(np.int32), oracle.bfs(g, d.source))
        else:
            np.testing.assert_array_equal(r.values[i], oracle.sssp(g, d.source))


def test_sssp_pair_condition_keeps_sparse_levels_scattering(grid_f32):
    """A 1024-slot group on a grid: with the pair condition a level gathers
    only when its estimated (edge, slot) pairs are worth a gather, so no more
    levels gather than with the edge condition alone; the distances are the
    oracle's either way."""
    g, graph = grid_f32
    src = np.resize(g.pick_sources(512, seed=143), 1024)
    ref, _ = oracle.batch("sssp", g, src[:512])
    gathers = {}
    for pr in (0.0, 0.5):
        r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src],
                          cgp.RunOptions(sssp_pull_edge_ratio=0.05, sssp_pull_pair_ratio=pr,
                                         profile_iterations=True), layout="query")
        v = r.values.view(np.float32)
        np.testing.assert_array_equal(v[:512], ref)
        np.testing.assert_array_equal(v[512:], ref)
        gathers[pr] = sum(p.sssp_mode == "pull" for p in r.iteration_profiles)
    assert gathers[0.0] > 0
    assert gathers[0.5] <= gathers[0.0]


@pytest.mark.parametrize("nq", [64, 128, 256, 300, 700, 1024])
@pytest.mark.parametrize("heavy", [0, 16, 1 << 20])
def test_sssp_gather_light_chunks(rmat_u32, nq, heavy):
    """Light vertices gathered in CTA chunks (up to 32 vertices / 2048 in-edges,
    a larger vertex alone; with heavy_degree 2^20 every vertex is light) give
    the same distances as one warp per vertex and as the oracle; groups wider
    than 256 slots (8 or 16 mask words, the last slice partly or wholly
    empty) are gathered in 256-slot slices."""
    g, graph = rmat_u32
    src = g.pick_sources(nq, seed=131)
    ref, _ = oracle.batch("sssp", g, src)
    descs = [cgp.QueryDescriptor(int(s), "sssp") for s in src]
    for chunks in (True, False):
        r = cgp.run_batch(graph, descs, cgp.RunOptions(traversal_mode="pull", heavy_degree=heavy,
                                                       light_chunks=chunks,
                                                       mask_words=nq // 64 if nq <= 256 else 0),
                          layout="query")
        np.testing.assert_array_equal(r.values, ref)


@pytest.mark.parametrize("ratio", [0.0, 0.05, 0.5])
def test_sssp_sliced_gather_grid_f32(grid_f32, ratio):
    """1024 f32 SSSP queries on a grid (16 mask words): the sliced chunked
    gather on whole-row and screened levels, mixed with scatter levels, gives
    the oracle's distances."""
    g, graph = grid_f32
    src = np.resize(g.pick_sources(512, seed=141), 1024)
    ref, _ = oracle.batch("sssp", g, src[:512])
    r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src],
                      cgp.RunOptions(sssp_pull_edge_ratio=ratio, sssp_pull_pair_ratio=0.0), layout="query")
    v = r.values.view(np.float32)
    np.testing.assert_array_equal(v[:512], ref)
    np.testing.assert_array_equal(v[512:], ref)



@pytest.mark.parametrize("loop", ["chunks", "device"])
@pytest.mark.parametrize("per_sync", [0, 1, 3])
def test_level_loop_forms_give_identical_results(rmat_u32, grid_f32, loop, per_sync):
    """Host-checked graph chunks and the device-looped graph (WHILE node on
    the done flag) give identical values on a shallow R-MAT and a deep grid,
    and BFS runs take the same levels and push/pull split (SSSP level counts
    may differ by a level between any two runs: relaxations within a level
    see each other's writes)."""
    for g, graph, kind in ((rmat_u32[0], rmat_u32[1], "bfs"), (rmat_u32[0], rmat_u32[1], "sssp"),
                           (grid_f32[0], grid_f32[1], "sssp")):
        src = g.pick_sources(70, seed=31)
        descs = [cgp.QueryDescriptor(int(s), kind) for s in src]
        r = cgp.run_batch(graph, descs, cgp.RunOptions(level_loop=loop, levels_per_sync=per_sync),
                          layout="query")
        ref, _ = oracle.batch(kind, g, src)
        np.testing.assert_array_equal(r.values.view(ref.dtype), ref)
        if kind == "bfs":
            base = cgp.run_batch(graph, descs, cgp.RunOptions(use_cuda_graph=False),
                                 layout="query")
            assert (r.iterations, r.push_levels, r.pull_levels) == \
                (base.iterations, base.push_levels, base.pull_levels)


def test_device_loop_honours_max_iterations(rmat_u32):
    g, graph = rmat_u32
    src = g.pick_sources(8, seed=32)
    r = cgp.run("bfs", graph, src, options=cgp.RunOptions(level_loop="device", max_iterations=2),
                layout="query")
    assert r.iterations == 2
    ref, _ = oracle.batch("bfs", g, src)
    v = r.values
    # depths 0..2 are final after two levels; deeper vertices are still unreached
    assert np.array_equal(np.where(ref <= 2, ref, INF), v)


def _with_paths(g, paths, length, wkind):
    """g plus `paths` disjoint paths of `length` vertices on new ids, with
    fresh symmetric weights: sources on a path keep tiny frontiers."""
    V = g.num_vertices
    u = np.repeat(np.arange(V), np.diff(g.row_offsets))
    keep = u < g.col_indices
    src = [u[keep]]
    dst = [g.col_indices[keep]]
    for p in range(paths):
        base = V + p * length
        src.append(np.arange(base, base + length - 1))
        dst.append(np.arange(base + 1, base + length))
    h = cgp.csr_from_edges(V + paths * length, np.concatenate(src), np.concatenate(dst))
    if wkind == "u32":
        return h.with_weights("u32", 1, 64, seed=7)
    return h.with_weights("f32", 1.0, 100.0, seed=7)


def _split_component_sources(g, n_big, n_small, seed):
    """n_big sources in the largest component, n_small outside it (vertices
    with edges): their chunks' frontiers stay small while the others grow."""
    lab = oracle.wcc_components(g).astype(np.int64)
    big = np.bincount(lab).argmax()
    deg = g.degrees()
    a = g.pick_sources(n_big, seed=seed, allowed=(lab == big).astype(np.uint8))
    b = g.pick_sources(n_small, seed=seed + 1, allowed=((lab != big) & (deg > 0)).astype(np.uint8))
    return np.concatenate([a, b])


@pytest.fixture(scope="module")
def rmat_paths():
    g = _with_paths(cgp.gen_rmat(12, 8, seed=101), 64, 40, "u32")
    return g, cgp.CsrGraph(g)


@pytest.fixture(scope="module")
def grid_paths():
    g = _with_paths(cgp.gen_grid(40, 50, 0.1, 0.01, seed=105), 32, 60, "f32")
    return g, cgp.CsrGraph(g)


@pytest.mark.parametrize("nq,kinds", [(64, "sssp"), (256, "sssp"), (200, "mixed"), (1024, "sssp")])
@pytest.mark.parametrize("ratio", [0.02, 0.3])
def test_sssp_direction_per_chunk(rmat_paths, nq, kinds, ratio):
    """SSSP gather/scatter chosen per 32-slot chunk: chunks whose sources lie
    on small path components keep scattering while the others gather in the
    same level; results stay exact."""
    g, graph = rmat_paths
    src = _split_component_sources(g, nq // 2, nq - nq // 2, seed=nq)
    if kinds == "mixed":
        descs = [cgp.QueryDescriptor(int(s), "bfs" if i % 3 == 0 else "sssp")
                 for i, s in enumerate(src)]
    else:
        descs = [cgp.QueryDescriptor(int(s), "sssp") for s in src]
    opts = cgp.RunOptions(sssp_chunk_direction=1, sssp_pull_edge_ratio=ratio, sssp_pull_pair_ratio=0.0, mask_words=16)
    r = cgp.run_batch(graph, descs, opts, layout="query")
    for i, d in enumerate(descs):
        exp = oracle.bfs(g, d.source).view(np.uint32) if d.kind == "bfs" else oracle.sssp(g, d.source)
        np.testing.assert_array_equal(r.values[i].view(np.uint32), exp)


def test_sssp_direction_per_chunk_f32_grid(grid_paths):
    g, graph = grid_paths
    src = _split_component_sources(g, 96, 32, seed=5)
    descs = [cgp.QueryDescriptor(int(s), "sssp") for s in src]
    for loop in ("chunks", "device"):
        r = cgp.run_batch(graph, descs, cgp.RunOptions(sssp_chunk_direction=1,
                                                       sssp_pull_edge_ratio=0.05, sssp_pull_pair_ratio=0.0,
                                                       level_loop=loop), layout="query")
        ref, _ = oracle.batch("sssp", g, src)
        np.testing.assert_array_equal(r.values.view(np.float32), ref)


@pytest.mark.parametrize("nq", [1, 64, 200, 256])
@pytest.mark.parametrize("depth", ["planes", "direct"])
@pytest.mark.parametrize("form", [1, 2])
def test_bfs_pull_form_options(rmat_u32, nq, depth, form):
    """The CTA-chunked light-vertex pull (form 1) and the lane pull in
    in-degree order (form 2, next masks of vertices without in-edges zeroed
    by k_clear_next) give the oracle's depths, with and without the
    in-degree 33..heavy kernel (heavy_degree 64 / 16)."""
    g, graph = rmat_u32
    src = g.pick_sources(nq, seed=90 + nq)
    ref, _ = oracle.batch("bfs", g, src)
    for ratio, heavy in ((0.01, 64), (0.2, 64), (0.05, 16)):
        r = _bfs(src, graph, cgp.RunOptions(bfs_pull_form=form, pull_edge_ratio=ratio,
                                            depth_mode=depth, heavy_degree=heavy))
        np.testing.assert_array_equal(r.values, ref)


def test_bfs_pull_in_degree_order_mixed_and_directed(rmat_u32):
    """Form 2 on a mixed BFS / k-hop / SSSP group and on a directed graph
    (pull over the transpose)."""
    g, graph = rmat_u32
    src = g.pick_sources(96, seed=97)
    descs = [cgp.QueryDescriptor(int(s), ["bfs", "khop", "sssp"][i % 3], 3)
             for i, s in enumerate(src)]
    r = cgp.run_heterogeneous(graph, cgp.HybridQueryBatch(descs),
                              options=cgp.RunOptions(bfs_pull_form=2, pull_edge_ratio=0.02),
                              layout="query")
    for i, d in enumerate(descs):
        if d.kind == "sssp":
            np.testing.assert_array_equal(r.values[i], oracle.sssp(g, d.source))
        else:
            exp = oracle.bfs(g, d.source, 3) if d.kind == "khop" else oracle.bfs(g, d.source)
            np.testing.assert_array_equal(r.values[i].view(np.int32), exp)
    rng = np.random.default_rng(98)
    V = 3000
    a = rng.integers(0, V, 24000)
    b = rng.integers(0, V, 24000)
    dg = cgp.csr_from_edges(V, a, b, symmetrize=False)
    dgraph = cgp.CsrGraph(dg)
    ds = dg.pick_sources(64, seed=99)
    ref, _ = oracle.batch("bfs", dg, ds)
    r = _bfs(ds, dgraph, cgp.RunOptions(bfs_pull_form=2, traversal_mode="pull"))
    np.testing.assert_array_equal(r.values, ref)
