"""Serving loop (continuous batching) against the oracle: every request's
result is the same alone and in the mix, whatever else shares the device."""
import threading
import time

import numpy as np
import pytest

import cgp_b200 as cgp
import oracle
from conftest import as_expected, host_csr

pytestmark = pytest.mark.gpu


def _case(golden, name):
    return next(c for c in golden["cases"] if c["name"] == name)


@pytest.fixture(scope="module")
def rmat():
    g = cgp.gen_rmat(12, 8, seed=201).with_weights("u32", 1, 64, seed=202)
    return g, cgp.CsrGraph(g)


def _expected(g, d):
    if d.kind == "bfs":
        return oracle.bfs(g, d.source).view(np.uint32)
    if d.kind == "khop":
        return oracle.bfs(g, d.source, d.k).view(np.uint32)
    if d.kind == "sssp":
        return oracle.sssp(g, d.source).view(np.uint32)
    return oracle.wcc_components(g)


def test_replenish_toy_like_validate_replenish(golden):
    c = _case(golden, "replenish_toy")
    g = host_csr(c["graph"])
    graph = cgp.CsrGraph(g)
    descs = [cgp.QueryDescriptor(s, k) for k, s in c["queries"]]
    r = cgp.run_replenish_pipeline(graph, descs, options=cgp.RunOptions(
        traversal_mode="push", enable_replenishment=True), slots=2)
    assert r.values.shape == (4, 4)
    for i, ((k, _), exp) in enumerate(zip(c["queries"], c["expect"])):
        if k == "sssp":
            np.testing.assert_array_equal(r.values[i], as_expected(exp, np.float32).view(np.uint32))
        else:
            np.testing.assert_array_equal(r.values[i].view(np.int32), np.asarray(exp, np.int32))
    assert all(q.state == "done" and q.completion_level > 0 for q in r.queries)
    # two slots for four queries: the second pair waited for a free slot
    assert max(q.admit_level for q in r.queries) > 0


@pytest.mark.parametrize("mode", ["push", "hybrid"])
def test_continuous_batching_matches_alone(rmat, mode):
    g, graph = rmat
    src = g.pick_sources(160, seed=5)
    kinds = ["bfs", "bfs", "sssp", "khop", "bfs", "sssp", "wcc", "bfs", "sssp", "khop"]
    descs = [cgp.QueryDescriptor(int(s), kinds[i % 10], 2 + i % 5) for i, s in enumerate(src)]
    outs = [np.full(g.num_vertices, 0xDEADBEEF, np.uint32) for _ in descs]
    with cgp.Server(graph, slots=16, options=cgp.RunOptions(traversal_mode=mode)) as s:
        tickets = []
        for i, (d, o) in enumerate(zip(descs, outs)):
            tickets.append(s.submit(d, o))
            if i % 7 == 0:
                time.sleep(0.002)  # arrivals while others are on the device
        s.drain(timeout_ms=120000)
        infos = [s.wait(t) for t in tickets]
        st = s.stats()
    assert st["completed"] == len(descs) and st["active_slots"] == 0
    for d, o, inf in zip(descs, outs, infos):
        assert inf.state == "done"
        np.testing.assert_array_equal(o, _expected(g, d))
    # the loop admitted requests while earlier ones were still running
    assert len({i.admit_level for i in infos}) > 1


def test_server_device_outputs_and_concurrent_submitters(rmat):
    import torch
    g, graph = rmat
    src = g.pick_sources(48, seed=9)
    descs = [cgp.QueryDescriptor(int(s), "bfs" if i % 2 else "sssp") for i, s in enumerate(src)]
    outs = [torch.empty(g.num_vertices, dtype=torch.int32, device="cuda") for _ in descs]
    with cgp.Server(graph, slots=8) as s:
        tickets = [None] * len(descs)

        def worker(lo, hi):
            for i in range(lo, hi):
                tickets[i] = s.submit(descs[i], outs[i])

        ts = [threading.Thread(target=worker, args=(k * 12, k * 12 + 12)) for k in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        s.drain(timeout_ms=120000)
        for t in tickets:
            assert s.wait(t).state == "done"
    for d, o in zip(descs, outs):
        np.testing.assert_array_equal(o.cpu().numpy().view(np.uint32), _expected(g, d))


def test_server_cancel(rmat):
    g, graph = rmat
    src = g.pick_sources(40, seed=11)
    descs = [cgp.QueryDescriptor(int(s), "sssp") for s in src]
    outs = [np.zeros(g.num_vertices, np.uint32) for _ in descs]
    with cgp.Server(graph, slots=4) as s:
        tickets = [s.submit(d, o) for d, o in zip(descs, outs)]
        for t in tickets[10:20]:
            s.cancel(t)
        s.drain(timeout_ms=120000)
        states = [s.poll(t).state for t in tickets]
    assert set(states[10:20]) <= {"cancelled", "done"}
    assert "cancelled" in states[10:20]
    for d, o, st in zip(descs, outs, states):
        if st == "done":
            np.testing.assert_array_equal(o, _expected(g, d))


def test_server_rejects_bad_requests(rmat):
    g, graph = rmat
    with cgp.Server(graph, slots=2) as s:
        with pytest.raises(ValueError):
            s.submit(cgp.QueryDescriptor(g.num_vertices, "bfs"))
        with pytest.raises(ValueError):
            s.submit(cgp.QueryDescriptor(0, "khop", -1))
        with pytest.raises(cgp.CgpError):
            s.poll(123456)


def test_server_slots_bounded_by_memory(rmat):
    g, graph = rmat
    V = g.num_vertices
    # room for roughly 8 slots' values plus the shared masks and staging
    budget = 3 * V * 8 * 2 + 3 * V * 4 + 32 * V * 4 + 8 * V * 4
    with cgp.Server(graph, slots=512, max_state_bytes=budget) as s:
        st = s.stats()
        assert 1 <= st["slots"] < 512 and st["state_bytes"] <= budget
        t = s.submit(cgp.QueryDescriptor(int(g.pick_sources(1, seed=3)[0]), "bfs"))
        assert s.wait(t, 60000).state == "done"


@pytest.mark.parametrize("policy,groups", [("chunks", 0), ("group", 0), ("group", 1),
                                           ("slots", 3), ("group", 4)])
def test_cohort_admission_matches_oracle(rmat, policy, groups):
    """Admission in whole 32-slot cohorts (requests enter only wholly free
    chunks) or group cohorts (only an empty group takes requests), over one
    or several traversal groups (uneven splits included), gives every request
    its exact result."""
    g, graph = rmat
    src = g.pick_sources(80, seed=61)
    kinds = ["bfs", "sssp", "khop"]
    descs = [cgp.QueryDescriptor(int(s), kinds[i % 3], 2 + i % 4 if i % 3 == 2 else 0)
             for i, s in enumerate(src)]
    outs = [np.zeros(g.num_vertices, np.uint32) for _ in descs]
    opts = cgp.RunOptions(serve_admission=policy, serve_groups=groups)
    with cgp.Server(graph, slots=64, options=opts) as s:
        tickets = [s.submit(d, o) for d, o in zip(descs, outs)]
        s.drain(timeout_ms=120000)
        assert all(s.poll(t).state == "done" for t in tickets)
        assert s.stats()["slots"] == 64
    for d, o in zip(descs, outs):
        np.testing.assert_array_equal(o, _expected(g, d))


def test_group_cohorts_overlap_staggered_arrivals():
    """Two groups under group cohorts: requests that arrive while a cohort
    runs in one group open a cohort in the other group, admitted before the
    first cohort finishes, and every request still gets its exact result.
    A 256 x 256 grid keeps the first (single-request) cohort running for
    hundreds of levels."""
    g = cgp.gen_grid(256, 256, 0.05, 0.0, seed=71).with_weights("u32", 1, 16, seed=72)
    graph = cgp.CsrGraph(g)
    src = g.pick_sources(25, seed=73)
    descs = [cgp.QueryDescriptor(int(s), "sssp" if i % 2 == 0 else "bfs")
             for i, s in enumerate(src)]
    outs = [np.zeros(g.num_vertices, np.uint32) for _ in descs]
    opts = cgp.RunOptions(serve_admission="group", serve_groups=2, levels_per_sync=1)
    with cgp.Server(graph, slots=64, options=opts) as s:
        first = s.submit(descs[0], outs[0])
        deadline = time.time() + 60
        while s.poll(first).state == "queued" and time.time() < deadline:
            time.sleep(0.0005)
        second = [s.submit(d, o) for d, o in zip(descs[1:], outs[1:])]
        s.drain(timeout_ms=120000)
        info1 = s.poll(first)
        infos2 = [s.poll(t) for t in second]
    assert all(i.state == "done" for i in [info1] + infos2)
    assert info1.slot < 32 and all(i.slot >= 32 for i in infos2)
    assert min(i.admit_ms for i in infos2) < info1.finish_ms
    for d, o in zip(descs, outs):
        np.testing.assert_array_equal(o, _expected(g, d))

@pytest.mark.parametrize("policy", ["slots", "group"])
def test_retire_mixes_device_host_and_discarded_outputs(rmat, policy):
    """Device outputs (written by the retire kernel itself), host outputs
    (through staging rows) and discarded results retire in the same passes;
    every kept result is exact."""
    import torch
    g, graph = rmat
    src = g.pick_sources(120, seed=71)
    kinds = ["bfs", "sssp", "khop"]
    descs = [cgp.QueryDescriptor(int(s), kinds[i % 3], 2 + i % 4 if i % 3 == 2 else 0)
             for i, s in enumerate(src)]
    outs = []
    for i in range(len(descs)):
        if (i // 3) % 3 == 0:  # output kinds cycle independently of query kinds
            outs.append(torch.zeros(g.num_vertices, dtype=torch.int32, device="cuda"))
        elif (i // 3) % 3 == 1:
            outs.append(np.zeros(g.num_vertices, np.uint32))
        else:
            outs.append(None)
    with cgp.Server(graph, slots=64, options=cgp.RunOptions(serve_admission=policy)) as s:
        tickets = [s.submit(d, o) for d, o in zip(descs, outs)]
        s.drain(timeout_ms=120000)
        assert all(s.poll(t).state == "done" for t in tickets)
    for d, o in zip(descs, outs):
        if o is None:
            continue
        got = o.cpu().numpy().view(np.uint32) if hasattr(o, "cpu") else o
        np.testing.assert_array_equal(got, _expected(g, d))
