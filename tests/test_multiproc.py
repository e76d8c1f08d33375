"""Multi-process host logic of the query-sharded path, on CPU with gloo
(world size 2).  The per-rank traversal is the CPU oracle here (the test
checks sharding, gathering and the reductions, not the kernels)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cgp_b200.parallel import shard_indices


def test_shard_indices_partition():
    for n in (0, 1, 7, 64, 257):
        for world in (1, 2, 3, 8):
            parts = [shard_indices(n, r, world) for r in range(world)]
            flat = sorted(i for p in parts for i in p)
            assert flat == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_indices(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    import torch.distributed as dist

    import cgp_b200 as cgp
    import oracle
    from cgp_b200.parallel import reduce_max, reduce_sum, run_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = cgp.gen_rmat(9, 8, seed=4).with_weights("u32", 1, 16, seed=5)
        src = g.pick_sources(11, seed=6)
        descs = [cgp.QueryDescriptor(int(s), "bfs" if i % 2 else "sssp") for i, s in enumerate(src)]

        class G:  # what run_sharded needs from a graph
            num_vertices = g.num_vertices

        def cpu_runner(_graph, local):
            rows = []
            for d in local:
                rows.append(oracle.bfs(g, d.source).view(np.uint32) if d.kind == "bfs"
                            else oracle.sssp(g, d.source))
            return np.stack(rows) if rows else np.zeros((0, g.num_vertices), np.uint32)

        full = run_sharded(G, descs, rank, world, runner=cpu_runner)
        t = reduce_max(float(rank + 1))
        s = reduce_sum(float(rank + 1))
        if rank == 0:
            exp = cpu_runner(None, descs)
            q.put((bool(np.array_equal(full, exp)), t, s))
    finally:
        dist.destroy_process_group()


def test_sharded_gather_and_reductions_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=180)
        assert p.exitcode == 0
    ok, t, s = q.get(timeout=10)
    assert ok
    assert t == 2.0 and s == 3.0


def _cuda_worker(rank, world, port, q):
    """One rank of the sharded path with the real CUDA runner: every rank
    runs its shard on cuda:0 (independent processes, no kernel waits on
    another) and rank 0 gathers the rows over gloo."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist

    import cgp_b200 as cgp
    import oracle
    from cgp_b200.parallel import run_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cgp.set_device(0)
        g = cgp.gen_rmat(12, 8, seed=14).with_weights("u32", 1, 16, seed=15)
        graph = cgp.CsrGraph(g)
        src = g.pick_sources(37, seed=16)
        descs = [cgp.QueryDescriptor(int(s), "bfs" if i % 3 else "sssp") for i, s in enumerate(src)]
        full = run_sharded(graph, descs, rank, world)
        if rank == 0:
            exp = np.stack([oracle.bfs(g, d.source).view(np.uint32) if d.kind == "bfs"
                            else oracle.sssp(g, d.source) for d in descs])
            q.put(bool(np.array_equal(full, exp)))
        else:
            assert full is None
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_cuda_runner_gloo_world2_one_gpu():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_cuda_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=300)
        assert p.exitcode == 0
    assert q.get(timeout=10)
