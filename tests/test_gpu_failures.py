"""Failure paths, injected on the host: a device allocation that fails (the
library's test hook makes its allocator report out-of-memory), waits that run
into their timeout, and a memory budget too small for one serving slot.  No
GPU fault is involved; after each failure the same objects must give exact
results again."""
import numpy as np
import pytest

import cgp_b200 as cgp
from cgp_b200 import _native as N
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture
def disarm():
    yield
    N.lib().cgp_debug_fail_allocations(-1)


def _bfs_sssp(g, n, seed):
    src = g.pick_sources(n, seed=seed)
    return src, ([cgp.QueryDescriptor(int(s), "bfs") for s in src[: n // 2]]
                 + [cgp.QueryDescriptor(int(s), "sssp") for s in src[n // 2:]])


def _expect(g, src, n):
    b, _ = oracle.batch("bfs", g, src[: n // 2])
    s, _ = oracle.batch("sssp", g, src[n // 2:])
    return np.concatenate([b.view(np.uint32), s.view(np.uint32)])


@pytest.mark.parametrize("after", [0, 1, 3, 6])
def test_injected_allocation_failure_then_clean_rerun(after, disarm):
    g = cgp.gen_rmat(12, 8, seed=401).with_weights("u32", 1, 32, seed=402)
    graph = cgp.CsrGraph(g)
    small_src, small = _bfs_sssp(g, 16, seed=403)
    # a first run leaves a cached workspace (and captured level graphs)
    r0 = cgp.run_batch(graph, small, layout="query")
    np.testing.assert_array_equal(r0.values.view(np.uint32), _expect(g, small_src, 16))
    big_src, big = _bfs_sssp(g, 300, seed=404)  # wider masks: buffers must grow
    N.check(N.lib().cgp_debug_fail_allocations(after))
    with pytest.raises(cgp.CgpOutOfMemory, match="injected"):
        cgp.run_batch(graph, big, layout="query")
    N.check(N.lib().cgp_debug_fail_allocations(-1))
    # the graph and its workspace pool stay usable, for both batch shapes
    r1 = cgp.run_batch(graph, small, layout="query")
    np.testing.assert_array_equal(r1.values.view(np.uint32), _expect(g, small_src, 16))
    r2 = cgp.run_batch(graph, big, layout="query")
    np.testing.assert_array_equal(r2.values.view(np.uint32), _expect(g, big_src, 300))


def test_injected_allocation_failure_in_graph_upload(disarm):
    g = cgp.gen_rmat(10, 8, seed=405)
    N.check(N.lib().cgp_debug_fail_allocations(1))
    with pytest.raises(cgp.CgpOutOfMemory):
        cgp.CsrGraph(g)
    N.check(N.lib().cgp_debug_fail_allocations(-1))
    graph = cgp.CsrGraph(g)
    src = g.pick_sources(8, seed=406)
    r = cgp.run("bfs", graph, src, layout="query")
    ref, _ = oracle.batch("bfs", g, src)
    np.testing.assert_array_equal(r.values, ref)


def test_injected_allocation_failure_in_server_create(disarm):
    g = cgp.gen_rmat(10, 8, seed=407)
    graph = cgp.CsrGraph(g)
    N.check(N.lib().cgp_debug_fail_allocations(2))
    with pytest.raises(cgp.CgpOutOfMemory):
        cgp.Server(graph, slots=8)
    N.check(N.lib().cgp_debug_fail_allocations(-1))
    d = cgp.QueryDescriptor(int(g.pick_sources(1, seed=408)[0]), "bfs")
    out = np.zeros(g.num_vertices, np.int32)
    with cgp.Server(graph, slots=8) as s:
        t = s.submit(d, out)
        assert s.wait(t, 60000).state == "done"
    np.testing.assert_array_equal(out, oracle.bfs(g, d.source))


def test_server_wait_and_drain_time_out_then_finish():
    g = cgp.gen_rmat(18, 16, seed=409).with_weights("u32", 1, 64, seed=410)
    graph = cgp.CsrGraph(g, symmetric=True)
    src = g.pick_sources(16, seed=411)
    descs = [cgp.QueryDescriptor(int(s), "sssp") for s in src]
    outs = [np.zeros(g.num_vertices, np.uint32) for _ in descs]
    with cgp.Server(graph, slots=16) as s:
        tickets = [s.submit(d, o) for d, o in zip(descs, outs)]
        with pytest.raises(cgp.CgpError) as ex:
            s.wait(tickets[-1], timeout_ms=1)
        assert ex.value.status == N.ERR_TIMEOUT
        with pytest.raises(cgp.CgpError) as ex:
            s.drain(timeout_ms=1)
        assert ex.value.status == N.ERR_TIMEOUT
        s.drain(timeout_ms=120000)
        assert all(s.wait(t, 1000).state == "done" for t in tickets)
    ref, _ = oracle.batch("sssp", g, src)
    np.testing.assert_array_equal(np.stack(outs), ref)


def test_server_budget_below_one_slot_is_rejected():
    g = cgp.gen_rmat(12, 8, seed=412)
    graph = cgp.CsrGraph(g)
    with pytest.raises(cgp.CgpOutOfMemory, match="one slot"):
        cgp.Server(graph, slots=64, max_state_bytes=4096)
    # a budget for a few slots admits a smaller server that still serves
    V = g.num_vertices
    with cgp.Server(graph, slots=64, max_state_bytes=3 * V * 8 + 3 * V * 4 + 40 * V * 4) as s:
        assert 1 <= s.stats()["slots"] < 64
        d = cgp.QueryDescriptor(int(g.pick_sources(1, seed=413)[0]), "bfs")
        out = np.zeros(V, np.int32)
        t = s.submit(d, out)
        assert s.wait(t, 60000).state == "done"
    np.testing.assert_array_equal(out, oracle.bfs(g, d.source))
