"""Parity on the shapes of the workloads the benchmark does not run itself:
a 4-neighbour grid with deletions and shortcuts, f32 weights U[1,100],
1024 SSSP queries (half from a corner region) plus one WCC; and a Chung-Lu
power-law graph (exponent 2.1, mean degree 16) with log-normal f32 weights,
4096 SSSP queries in four 1024-slot groups (half from the top 1% of hubs)
plus one WCC.  Reduced vertex counts keep the CPU oracle within seconds; the
full-size grid is checked by optimality certificates on the device."""
import numpy as np
import pytest

import cgp_b200 as cgp
import oracle

pytestmark = pytest.mark.gpu


def _corner_and_uniform(g, rows, cols, n, seed):
    corner = np.zeros(g.num_vertices, np.uint8)
    r = np.arange(g.num_vertices) // cols
    c = np.arange(g.num_vertices) % cols
    corner[(r < max(2, rows // 10)) & (c < max(2, cols // 10))] = 1
    a = g.pick_sources(n // 2, seed=seed, allowed=corner)
    b = g.pick_sources(n - n // 2, seed=seed + 1)
    return np.concatenate([a, b])


def _check_hetero(g, graph, sources, opts):
    descs = [cgp.QueryDescriptor(int(s), "sssp") for s in sources] + [cgp.QueryDescriptor(0, "wcc")]
    r = cgp.run_heterogeneous(graph, cgp.HybridQueryBatch(descs), options=opts, layout="query")
    ref, _ = oracle.batch("sssp", g, sources)
    np.testing.assert_array_equal(r.values[:-1].view(np.float32), ref)
    np.testing.assert_array_equal(r.values[-1], oracle.wcc_components(g))
    return r


@pytest.mark.parametrize("mode", ["hybrid", "push"])
def test_grid_1024_sssp_plus_wcc(mode):
    rows, cols = 96, 96
    g = cgp.gen_grid(rows, cols, 0.1, 0.001, seed=201).with_weights("f32", 1.0, 100.0, seed=202)
    graph = cgp.CsrGraph(g)
    src = _corner_and_uniform(g, rows, cols, 1024, seed=203)
    r = _check_hetero(g, graph, src, cgp.RunOptions(traversal_mode=mode))
    assert r.mask_words == 16
    assert r.iterations > 30  # deep traversal: many captured level chunks


def test_chung_lu_4096_sssp_in_four_groups_plus_wcc():
    g = cgp.gen_chung_lu(1 << 14, 2.1, 16.0, seed=211).with_weights("f32", 0.0, 1.0, seed=212,
                                                                    lognormal=True)
    graph = cgp.CsrGraph(g)
    deg = g.degrees()
    hubs = np.zeros(g.num_vertices, np.uint8)
    hubs[np.argsort(-deg)[: max(1, g.num_vertices // 100)]] = 1
    a = g.pick_sources(2048, seed=213, allowed=hubs)
    b = g.pick_sources(2048, seed=214)
    src = np.concatenate([a, b])
    r = _check_hetero(g, graph, src, cgp.RunOptions(mask_words=16))
    assert r.groups == 4


@pytest.mark.parametrize("mode", ["hybrid", "push", "pull"])
def test_c1_rmat16_64_bfs_every_column(mode):
    """The CPU-runnable workload at its own shape: R-MAT 16, edge factor 16,
    64 BFS sources from non-isolated vertices, one 64-bit mask word; every
    column compared with the CPU oracle."""
    g = cgp.gen_rmat(16, 16, 0.57, 0.19, 0.19, seed=1)
    graph = cgp.CsrGraph(g)
    src = g.pick_sources(64, seed=42)
    r = cgp.run("bfs", graph, src, options=cgp.RunOptions(traversal_mode=mode), layout="query")
    assert r.mask_words == 1
    ref, _ = oracle.batch("bfs", g, src)
    np.testing.assert_array_equal(r.values, ref)


def _certificate_f32(out, src, g, dev, chunk=1 << 16):
    """d[src] = 0; d[v] <= fl(d[u] + w) for every edge with u reached; every
    reached v != src has an edge with equality (fp32 round to nearest, the
    kernels' __fadd_rn)."""
    import torch
    V, Q = out.shape
    row = torch.from_numpy(g.row_offsets).to(dev)
    col = torch.from_numpy(g.col_indices.astype(np.int64)).to(dev)
    w = torch.from_numpy(g.weights).to(dev)
    u_of = torch.repeat_interleave(torch.arange(V, device=dev), row[1:] - row[:-1])
    q = torch.arange(Q, device=dev)
    s = torch.as_tensor(np.asarray(src), device=dev).long()
    assert bool((out[s, q] == 0).all())
    tight = torch.zeros((V, Q), dtype=torch.int32, device=dev)
    for e0 in range(0, col.numel(), chunk):
        u = u_of[e0:e0 + chunk]
        v = col[e0:e0 + chunk]
        du = out[u]
        dv = out[v]
        cand = du + w[e0:e0 + chunk].unsqueeze(1)
        ru = torch.isfinite(du)
        assert bool((~ru | (dv <= cand)).all())
        tight.index_reduce_(0, v, (ru & (dv == cand)).to(torch.int32), "amax")
        del du, dv, cand, ru
    reached = torch.isfinite(out)
    assert bool((~reached | (out == 0) | (tight > 0)).all())


def _certificate_bfs(out, src, g, dev, chunk=1 << 18):
    """d[src] = 0; for every edge u-v |d[u] - d[v]| <= 1 with both reached or
    both unreached; every reached v != src has a neighbour at d[v] - 1."""
    import torch
    V, Q = out.shape
    row = torch.from_numpy(g.row_offsets).to(dev)
    col = torch.from_numpy(g.col_indices.astype(np.int64)).to(dev)
    u_of = torch.repeat_interleave(torch.arange(V, device=dev), row[1:] - row[:-1])
    q = torch.arange(Q, device=dev)
    s = torch.as_tensor(np.asarray(src), device=dev).long()
    assert bool((out[s, q] == 0).all())
    inf = 2**31 - 1
    parent = torch.zeros((V, Q), dtype=torch.int32, device=dev)
    for e0 in range(0, col.numel(), chunk):
        du = out[u_of[e0:e0 + chunk]].long()
        v = col[e0:e0 + chunk]
        dv = out[v].long()
        ru, rv = du != inf, dv != inf
        assert bool((ru == rv).all())
        assert bool((~ru | ((du - dv).abs() <= 1)).all())
        parent.index_reduce_(0, v, (ru & (du == dv - 1)).to(torch.int32), "amax")
        del du, dv, ru, rv
    reached = out != inf
    assert bool((~reached | (out == 0) | (parent > 0)).all())


@pytest.mark.slow
def test_grid_2048_full_size_certificate():
    """Full-size grid (2048 x 2048, V = 4.19M), 1024 f32 SSSP queries, checked
    by the optimality conditions in fp32 (same rounding as the kernels'
    __fadd_rn): d[src] = 0; d[v] <= fl(d[u] + w) for every edge with u
    reached; every reached v != src has an edge with equality."""
    import torch
    rows = cols = 2048
    g = cgp.gen_grid(rows, cols, 0.1, 0.001, seed=221).with_weights("f32", 1.0, 100.0, seed=222)
    graph = cgp.CsrGraph(g)
    src = _corner_and_uniform(g, rows, cols, 1024, seed=223)
    dev = torch.device("cuda", 0)
    out = torch.empty((g.num_vertices, 1024), dtype=torch.float32, device=dev)
    r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), "sssp") for s in src], out=out)
    assert r.mask_words == 16
    _certificate_f32(out, src, g, dev)
    # a few full columns against the CPU oracle
    for k in (0, 700):
        np.testing.assert_array_equal(out[:, k].cpu().numpy(), oracle.sssp(g, int(src[k])))
    del out
    # the WCC pass of the same workload, every label against union-find on the CPU
    lab = cgp.run("wcc", graph, [0]).values[:, 0]
    np.testing.assert_array_equal(lab.view(np.uint32), oracle.wcc_components(g))


@pytest.mark.slow
def test_chung_lu_full_size_1024_slot_groups_certificate():
    """The large heterogeneous workload at its own size: Chung-Lu with 2^25
    vertices (exponent 2.1, mean degree 16, ~537M CSR entries), log-normal f32
    weights, one 1024-slot SSSP group and one 1024-slot BFS group (half of the
    sources among the top 1% of hubs), each written in place into a 137 GB
    device output.  64 columns of each group are checked by the optimality
    conditions on the device and one column of each against the CPU oracle;
    the WCC pass against union-find."""
    import torch
    V = 1 << 25
    g = cgp.gen_chung_lu(V, 2.1, 16.0, seed=1).with_weights("f32", 0.0, 1.0, seed=2,
                                                            lognormal=True)
    graph = cgp.CsrGraph(g, symmetric=True)
    dev = torch.device("cuda", 0)
    deg = g.degrees()
    hubs = np.zeros(V, np.uint8)
    hubs[np.argsort(-deg, kind="stable")[: V // 100]] = 1
    src = np.concatenate([g.pick_sources(512, seed=231, allowed=hubs),
                          g.pick_sources(512, seed=232)])
    cols = np.r_[0:32, 512:544]
    opts = cgp.RunOptions(mask_words=16, depth_mode="direct")
    for kind in ("sssp", "bfs"):
        out = torch.empty((V, 1024), dtype=torch.float32 if kind == "sssp" else torch.int32,
                          device=dev)
        r = cgp.run_batch(graph, [cgp.QueryDescriptor(int(s), kind) for s in src], opts, out=out)
        assert r.mask_words == 16 and r.groups == 1
        sub = out[:, torch.as_tensor(cols, device=dev)].clone()
        one = out[:, 600].cpu().numpy()
        del out, r  # the result holds the output tensor too
        torch.cuda.empty_cache()
        if kind == "sssp":
            _certificate_f32(sub, src[cols], g, dev, chunk=1 << 20)
            np.testing.assert_array_equal(one, oracle.sssp(g, int(src[600])))
        else:
            _certificate_bfs(sub, src[cols], g, dev, chunk=1 << 20)
            np.testing.assert_array_equal(one, oracle.bfs(g, int(src[600])))
        del sub
        torch.cuda.empty_cache()
    lab = cgp.run("wcc", graph, [0]).values[:, 0]
    np.testing.assert_array_equal(lab.view(np.uint32), oracle.wcc_components(g))
