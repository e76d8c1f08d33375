"""Multi-GPU query sharding (one process per GPU).

Queries are independent, so every rank holds a replica of the CSR and runs
its own shard of the batch; there is no collective on the data path.  The
only communication is at the end: timing (max over ranks), counts (sum) and,
when asked, gathering the per-rank result rows to rank 0 as tensors through
torch.distributed (NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def shard_indices(n: int, rank: int, world: int) -> list[int]:
    """Round-robin shard of n queries for `rank` (balanced to within one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return list(range(rank, n, world))


def _gather_rows(local: np.ndarray, n: int, V: int, rank: int, world: int):
    """Gathers every rank's [n_local, V] uint32 rows to rank 0 as one
    [n, V] array in submission order (rows padded to the largest shard so
    that every rank sends a tensor of the same shape)."""
    import torch
    import torch.distributed as dist
    n_max = (n + world - 1) // world
    on_gpu = dist.get_backend() == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
    buf = torch.zeros((n_max, V), dtype=torch.int32, device=dev)
    if len(local):
        buf[:len(local)] = torch.from_numpy(np.ascontiguousarray(local).view(np.int32)).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, parts, dst=0)
    if rank != 0:
        return None
    out = np.zeros((n, V), np.uint32)
    for r in range(world):
        ids = shard_indices(n, r, world)
        if ids:
            out[np.asarray(ids)] = parts[r][:len(ids)].cpu().numpy().view(np.uint32)
    return out


def run_sharded(graph, descs: Sequence, rank: int, world: int,
                runner: Callable | None = None, gather: bool = True):
    """Runs this rank's shard of `descs` and (optionally) gathers the
    query-major result rows to rank 0 in submission order.

    runner(graph, local_descs) -> array [n_local, V]; defaults to the CUDA
    path (cgp_b200.run_batch with a query-major layout).  Returns the full
    [N, V] array on rank 0 when gathering (None on the other ranks), else the
    local rows."""
    idx = shard_indices(len(descs), rank, world)
    if runner is None:
        from .api import run_batch

        def runner(g, d):
            return run_batch(g, d, layout="query").values
    V = graph.num_vertices
    local = runner(graph, [descs[i] for i in idx]) if idx else np.zeros((0, V), np.uint32)
    local = np.ascontiguousarray(local).view(np.uint32)
    if not gather or world == 1:
        return local
    return _gather_rows(local, len(descs), V, rank, world)


def reduce_max(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def reduce_sum(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.item()
