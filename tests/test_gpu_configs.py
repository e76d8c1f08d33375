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
    row = torch.from_numpy(g.row_offsets).to(dev)
    col = torch.from_numpy(g.col_indices.astype(np.int64)).to(dev)
    w = torch.from_numpy(g.weights).to(dev)
    u_of = torch.repeat_interleave(torch.arange(g.num_vertices, device=dev), row[1:] - row[:-1])
    q = torch.arange(1024, device=dev)
    s = torch.as_tensor(src, device=dev).long()
    assert bool((out[s, q] == 0).all())
    tight = torch.zeros((g.num_vertices, 1024), dtype=torch.int32, device=dev)
    chunk = 1 << 16
    for e0 in range(0, col.numel(), chunk):
        u = u_of[e0:e0 + chunk]
        v = col[e0:e0 + chunk]
        du = out[u]
        dv = out[v]
        cand = du + w[e0:e0 + chunk].unsqueeze(1)  # fp32, round to nearest
        ru = torch.isfinite(du)
        assert bool((~ru | (dv <= cand)).all())
        tight.index_reduce_(0, v, (ru & (dv == cand)).to(torch.int32), "amax")
        del du, dv, cand, ru
    reached = torch.isfinite(out)
    is_src = out == 0
    assert bool((~reached | is_src | (tight > 0)).all())
    # a few full columns against the CPU oracle
    for k in (0, 700):
        np.testing.assert_array_equal(out[:, k].cpu().numpy(), oracle.sssp(g, int(src[k])))
