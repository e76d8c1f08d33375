"""cgp_bfs_batch_noalloc: the batched BFS for callers that cannot allocate
device memory (a framework that reserved the memory pool up front, latency
paths where cudaMalloc/cudaFree would stall the device, hosts that only lend
their own buffers).  The entry point must give exactly the depths of the
regular entry point (cgp_batch_run) while allocating nothing; it is called
twice in a row to show that the shared scratch array is reset between calls.

This file is collected last on purpose (tests/test_zz_*)."""
import ctypes

import numpy as np
import pytest

import cgp_b200 as cgp
from cgp_b200 import _native as N

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    f = N.lib().cgp_bfs_batch_noalloc
    f.restype = ctypes.c_int32
    f.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                  ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
    return f


def _run_noalloc(f, row_d, col_d, V, E, sources, out_d, symmetric, stream):
    src = np.ascontiguousarray(sources, np.int32)
    ob = row_d.element_size()
    st = f(row_d.data_ptr(), ob, col_d.data_ptr(), V, E, src.ctypes.data, len(src), symmetric,
           out_d.data_ptr(), stream)
    N.check(st, "cgp_bfs_batch_noalloc")


# (queries, symmetric, offset bytes): one, two and four mask words; 32- and
# 64-bit row offsets
@pytest.mark.parametrize("nq,symmetric,ob", [(64, 1, 4), (200, 0, 4), (100, 1, 8), (30, 0, 8)])
def test_noalloc_matches_regular_entry_point_twice(nq, symmetric, ob):
    import torch
    g = cgp.gen_rmat(14, 8, seed=301)
    V, E = g.num_vertices, g.num_edges
    dev = torch.device("cuda", 0)
    row_d = torch.from_numpy(g.row_offsets.astype(np.int32 if ob == 4 else np.int64)).to(dev)
    col_d = torch.from_numpy(g.col_indices).to(dev)
    graph = cgp.CsrGraph(g)
    f = _noalloc_fn()
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        src = g.pick_sources(nq, seed=310 + call)
        expect = cgp.run("bfs", graph, src).values  # regular entry point, [V, nq]
        out = torch.full((V, nq), -7, dtype=torch.int32, device=dev)
        free_before = torch.cuda.mem_get_info(dev)[0]
        _run_noalloc(f, row_d, col_d, V, E, src, out, symmetric, stream)
        torch.cuda.synchronize(dev)
        if call == 1:  # the first call may have loaded the library's device module
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        np.testing.assert_array_equal(out.cpu().numpy(), expect)


def test_noalloc_rejects_oversized_graph_and_bad_input():
    import torch
    dev = torch.device("cuda", 0)
    f = _noalloc_fn()
    V = 1_000_000  # 36 B/vertex needs ~36 MB > 24 MiB
    row_d = torch.zeros(V + 1, dtype=torch.int32, device=dev)
    col_d = torch.zeros(1, dtype=torch.int32, device=dev)
    out = torch.zeros((V, 1), dtype=torch.int32, device=dev)
    st = f(row_d.data_ptr(), 4, col_d.data_ptr(), V, 0, np.zeros(1, np.int32).ctypes.data, 1, 1,
           out.data_ptr(), None)
    assert st == N.ERR_INVALID_ARG
    assert "scratch" in N.last_error()
    # a column outside [0, V) is caught on the device before any traversal
    row = torch.tensor([0, 1, 1], dtype=torch.int32, device=dev)
    col = torch.tensor([5], dtype=torch.int32, device=dev)
    out2 = torch.zeros((2, 1), dtype=torch.int32, device=dev)
    st = f(row.data_ptr(), 4, col.data_ptr(), 2, 1, np.zeros(1, np.int32).ctypes.data, 1, 1,
           out2.data_ptr(), None)
    assert st == N.ERR_INVALID_ARG and "malformed" in N.last_error()
