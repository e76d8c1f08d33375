"""cgp_b200: B200-native concurrent multi-query graph traversal.

Many BFS, SSSP, k-hop BFS and WCC queries over one CSR graph, each vertex
carrying a query bitmask; hand-written sm_100a kernels behind the C ABI in
include/cgp_b200.h (library: cgp_b200/libcgp_b200.so).
"""
from ._native import (BFS_UNREACHED, U32_UNREACHED, CgpError, CgpInvalidArgument,  # noqa: F401
                      CgpOutOfMemory, declared_symbols, lib)
from .api import (CsrGraph, Enactor, HostCsr, HybridQueryBatch, IterationProfile,  # noqa: F401
                  QueryBatch, QueryDescriptor, RunOptions, RunResult, csr_from_edges,
                  gen_chung_lu, gen_grid, gen_rmat, load_binary_csr, load_galois_gr,
                  load_matrix_market, run, run_batch, run_heterogeneous, set_device,
                  Server, RequestInfo, run_replenish_pipeline, autotune)

__all__ = [
    "CsrGraph", "Enactor", "HostCsr", "HybridQueryBatch", "IterationProfile", "QueryBatch",
    "QueryDescriptor", "RunOptions", "RunResult", "csr_from_edges", "gen_chung_lu", "gen_grid",
    "gen_rmat", "load_binary_csr", "load_galois_gr", "load_matrix_market", "run", "run_batch",
    "run_heterogeneous", "set_device", "Server", "RequestInfo", "run_replenish_pipeline",
    "autotune", "BFS_UNREACHED", "U32_UNREACHED", "CgpError", "CgpInvalidArgument",
    "CgpOutOfMemory", "declared_symbols", "lib",
]
