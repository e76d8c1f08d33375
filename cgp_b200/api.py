"""Host-side mirror of the reference's query/operator interface over the C ABI.

Names follow puercgp (puercgp/include/puercgp/...):
  run(policy, graph, queries, context, options)   -> run.hxx:11-23
  run_heterogeneous(graph, batch, context, options) -> hybrid_engine.hxx:1144-1150
  RunOptions                                      -> core/types.hxx:26-46
  QueryDescriptor / HybridQueryBatch / QueryBatch -> core/query_descriptor.hxx, core/query_batch.hxx
  RunResult / IterationProfile                    -> core/result.hxx
  Enactor (problem/enactor/advance+filter)        -> cgp/include/gunrock/framework/{problem,enactor}.hxx
Invalid batches raise ValueError where the reference throws std::invalid_argument.
"""
from __future__ import annotations

import ctypes
import dataclasses
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _native as N

POLICIES = {"bfs": N.KIND_BFS, "sssp": N.KIND_SSSP, "wcc": N.KIND_WCC, "khop": N.KIND_KHOP}
MODES = {"push": N.MODE_PUSH, "pull": N.MODE_PULL, "hybrid": N.MODE_HYBRID}


# ------------------------------------------------------------------ inputs
@dataclass
class HostCsr:
    """Host CSR graph: int64 row offsets, int32 columns, optional weights."""
    row_offsets: np.ndarray
    col_indices: np.ndarray
    weights: np.ndarray | None = None

    @property
    def num_vertices(self) -> int:
        return len(self.row_offsets) - 1

    @property
    def num_edges(self) -> int:
        return len(self.col_indices)

    @property
    def weight_kind(self) -> int:
        if self.weights is None:
            return N.WEIGHT_NONE
        return N.WEIGHT_F32 if self.weights.dtype == np.float32 else N.WEIGHT_U32

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_offsets)

    def _as_c(self) -> N.CgpHostCsr:
        c = N.CgpHostCsr()
        c.num_vertices = self.num_vertices
        c.num_edges = self.num_edges
        self._keep = (np.ascontiguousarray(self.row_offsets, np.int64),
                      np.ascontiguousarray(self.col_indices, np.int32))
        c.row_offsets = self._keep[0].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        c.col_indices = self._keep[1].ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        c.weights = None
        c.weight_kind = N.WEIGHT_NONE
        return c

    def with_weights(self, kind: str, p0: float, p1: float, seed: int = 2,
                     lognormal: bool = False) -> "HostCsr":
        """Symmetric seeded weights: kind 'u32' uniform ints in [p0, p1];
        'f32' uniform reals in [p0, p1), or exp(p0 + p1*N(0,1)) if lognormal."""
        c = self._as_c()
        wk = N.WEIGHT_U32 if kind == "u32" else N.WEIGHT_F32
        N.check(N.lib().cgp_gen_weights(ctypes.byref(c), wk, p0, p1, int(lognormal), seed),
                "cgp_gen_weights")
        dt = np.uint32 if wk == N.WEIGHT_U32 else np.float32
        buf = (ctypes.c_char * (4 * self.num_edges)).from_address(c.weights) if self.num_edges else b""
        w = np.frombuffer(bytes(buf), dtype=dt).copy() if self.num_edges else np.zeros(0, dt)
        c.row_offsets = ctypes.POINTER(ctypes.c_int64)()  # not owned by the library
        c.col_indices = ctypes.POINTER(ctypes.c_int32)()
        N.lib().cgp_host_csr_free(ctypes.byref(c))
        return HostCsr(self.row_offsets, self.col_indices, w)

    def pick_sources(self, count: int, seed: int = 42, min_degree: int = 1,
                     allowed: np.ndarray | None = None) -> np.ndarray:
        c = self._as_c()
        out = np.zeros(count, np.int32)
        al = None
        if allowed is not None:
            allowed = np.ascontiguousarray(allowed, np.uint8)
            al = allowed.ctypes.data
        N.check(N.lib().cgp_pick_sources(ctypes.byref(c), count, min_degree, al, seed,
                                         out.ctypes.data), "cgp_pick_sources")
        return out


def _take_csr(c: N.CgpHostCsr) -> HostCsr:
    V, E = c.num_vertices, c.num_edges
    row = np.ctypeslib.as_array(c.row_offsets, shape=(V + 1,)).copy()
    col = np.ctypeslib.as_array(c.col_indices, shape=(max(E, 1),))[:E].copy()
    w = None
    if c.weights and c.weight_kind != N.WEIGHT_NONE:
        dt = np.uint32 if c.weight_kind == N.WEIGHT_U32 else np.float32
        w = np.frombuffer((ctypes.c_char * (4 * max(E, 1))).from_address(c.weights), dtype=dt)[:E].copy()
    N.lib().cgp_host_csr_free(ctypes.byref(c))
    return HostCsr(row, col, w)


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, seed: int = 1, permute: bool = True) -> HostCsr:
    """Seeded R-MAT graph, symmetrised, deduplicated, self loops removed."""
    h = N.CgpHostCsr()
    N.check(N.lib().cgp_gen_rmat(scale, edge_factor, a, b, c, seed, int(permute), ctypes.byref(h)),
            "cgp_gen_rmat")
    return _take_csr(h)


def gen_grid(rows: int, cols: int, delete_frac: float = 0.1, shortcut_frac: float = 0.001,
             seed: int = 1) -> HostCsr:
    h = N.CgpHostCsr()
    N.check(N.lib().cgp_gen_grid(rows, cols, delete_frac, shortcut_frac, seed, ctypes.byref(h)),
            "cgp_gen_grid")
    return _take_csr(h)


def gen_chung_lu(num_vertices: int, exponent: float = 2.1, mean_degree: float = 16.0,
                 seed: int = 1) -> HostCsr:
    h = N.CgpHostCsr()
    N.check(N.lib().cgp_gen_chung_lu(num_vertices, exponent, mean_degree, seed, ctypes.byref(h)),
            "cgp_gen_chung_lu")
    return _take_csr(h)


def csr_from_edges(num_vertices: int, src: Sequence[int], dst: Sequence[int],
                   symmetrize: bool = True) -> HostCsr:
    s = np.ascontiguousarray(src, np.int32)
    d = np.ascontiguousarray(dst, np.int32)
    h = N.CgpHostCsr()
    N.check(N.lib().cgp_csr_from_edges(num_vertices, len(s), s.ctypes.data, d.ctypes.data,
                                       int(symmetrize), ctypes.byref(h)), "cgp_csr_from_edges")
    return _take_csr(h)


def load_matrix_market(path: str) -> HostCsr:
    """Matrix Market with the reference loader's semantics (mtx_loader.hxx:99-187)."""
    h = N.CgpHostCsr()
    N.check(N.lib().cgp_load_matrix_market(str(path).encode(), ctypes.byref(h)),
            "cgp_load_matrix_market")
    return _take_csr(h)


def load_binary_csr(path: str) -> HostCsr:
    """csr_vlist.bin / csr_elist.bin / csr_weightlist.bin directory (mtx_loader.hxx:189-260)."""
    h = N.CgpHostCsr()
    N.check(N.lib().cgp_load_binary_csr(str(path).encode(), ctypes.byref(h)),
            "cgp_load_binary_csr")
    return _take_csr(h)


def load_galois_gr(path: str, read_edge_data: bool = False) -> HostCsr:
    """Galois .gr version 1 (load_gr, cgp/examples/algorithms/bfs/cgp_bfs.cu:215-260):
    topology only like the reference, or with 4-byte edge data as uint32
    weights when read_edge_data is set."""
    h = N.CgpHostCsr()
    N.check(N.lib().cgp_load_galois_gr(str(path).encode(), int(read_edge_data), ctypes.byref(h)),
            "cgp_load_galois_gr")
    return _take_csr(h)


def set_device(device: int) -> None:
    """Selects the CUDA device of this thread's subsequent library calls."""
    N.check(N.lib().cgp_set_device(int(device)), "cgp_set_device")


class CsrGraph:
    """Device-resident CSR graph (csr_graph_storage, csr_graph.hxx:42-75)."""

    def __init__(self, host: HostCsr, offsets64: bool = False, symmetric: bool | None = None):
        self.host = host
        row = np.ascontiguousarray(host.row_offsets, np.int64)
        col = np.ascontiguousarray(host.col_indices, np.int32)
        w = None if host.weights is None else np.ascontiguousarray(host.weights)
        flags = (N.GRAPH_OFFSETS64 if offsets64 else 0) | (N.GRAPH_SYMMETRIC if symmetric else 0)
        h = ctypes.c_void_p()
        N.check(N.lib().cgp_graph_create(row.ctypes.data, 8, col.ctypes.data,
                                         None if w is None else w.ctypes.data, host.weight_kind,
                                         host.num_vertices, host.num_edges, flags,
                                         ctypes.byref(h)), "cgp_graph_create")
        self._h = h
        V, E, wk, sym = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
        N.check(N.lib().cgp_graph_info(h, ctypes.byref(V), ctypes.byref(E), ctypes.byref(wk),
                                       ctypes.byref(sym)))
        self.num_vertices, self.num_edges = V.value, E.value
        self.weight_kind, self.symmetric = wk.value, bool(sym.value)

    @property
    def handle(self):
        return self._h

    def get_number_of_vertices(self) -> int:
        return self.num_vertices

    def get_number_of_edges(self) -> int:
        return self.num_edges

    def close(self):
        if getattr(self, "_h", None):
            N.lib().cgp_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ queries
@dataclass
class QueryDescriptor:
    """query_descriptor_t (query_descriptor.hxx:19-24) + k for k-hop BFS."""
    source: int = 0
    kind: str = "bfs"
    k: int = 0


class QueryBatch:
    """query_batch<int> (core/query_batch.hxx): sources of one policy."""

    def __init__(self, sources: Iterable[int]):
        self.sources = [int(s) for s in sources]

    def __len__(self):
        return len(self.sources)

    def validate(self, max_queries: int = 0) -> None:
        if not self.sources:
            raise ValueError("query_batch must contain at least one source")
        if max_queries and len(self.sources) > max_queries:
            raise ValueError("query_batch exceeds max_queries")
        if any(s < 0 for s in self.sources):
            raise ValueError("query_batch sources must be non-negative")


class HybridQueryBatch:
    """hybrid_query_batch (query_descriptor.hxx:28-145).  The reference caps a
    batch at 64 queries (one uint64 mask); here a batch of any size runs in
    groups of up to 1024 (16 mask words)."""

    def __init__(self, descs: Iterable[QueryDescriptor]):
        self.descs = list(descs)

    def __len__(self):
        return len(self.descs)

    def validate(self, max_queries: int = 0) -> None:
        if not self.descs:
            raise ValueError("hybrid_query_batch must be non-empty")
        if max_queries and len(self.descs) > max_queries:
            raise ValueError("hybrid_query_batch exceeds max_queries")
        for d in self.descs:
            if d.source < 0:
                raise ValueError("query source must be non-negative")
            if d.kind not in POLICIES:
                raise ValueError(f"unknown query kind {d.kind!r}")

    def bfs_slot_mask(self) -> int:
        return sum(1 << i for i, d in enumerate(self.descs) if d.kind in ("bfs", "khop"))

    def nonbfs_slot_mask(self) -> int:
        return sum(1 << i for i, d in enumerate(self.descs) if d.kind not in ("bfs", "khop"))

    def has_bfs(self) -> bool:
        return any(d.kind == "bfs" for d in self.descs)

    def has_wcc(self) -> bool:
        return any(d.kind == "wcc" for d in self.descs)


@dataclass
class RunOptions:
    """run_options (core/types.hxx:26-46) plus the B200 execution knobs."""
    traversal_mode: str = "hybrid"
    push_strategy: str = "edge_balanced"
    pull_strategy: str = "bitmap"
    pull_frontier_ratio: float = 0.15
    pull_edge_ratio: float = 0.20
    profile_iterations: bool = False
    emit_nvtx: bool = False
    max_iterations: int = 0
    max_queries: int = 0
    enable_replenishment: bool = False
    discard_results: bool = False
    use_cuda_graph: bool = True
    levels_per_sync: int = 0
    mask_words: int = 0
    depth_mode: str = "auto"
    heavy_degree: int = 0
    profile_kernels: bool = False
    dense_unroll: int = 0
    sssp_pull_edge_ratio: float = 0.5
    sssp_pull_pair_ratio: float = 0.5  # gather also needs est. pairs >= ratio * E * SSSP chunks
    light_chunks: bool = True
    level_loop: str = "auto"    # "auto", "chunks" (host-checked graph chunks), "device"
    sssp_chunk_direction: int = 0  # 1 per 32-slot chunk, -1 whole group, 0 auto (serving: chunk)
    bfs_pull_chunks: bool = False  # CTA-chunked light-vertex BFS pull on levels that read most edges
    bfs_pull_form: int = 0  # 0 lane per vertex (vertex order), 1 CTA chunks, 2 lane per vertex
                            # in decreasing in-degree order (bfs_pull_chunks=True means 1)
    serve_admission: str = "slots"  # serving: "slots" (any free slot), "chunks" (whole 32-slot
                                    # cohorts) or "group" (a new cohort only in an empty group)
    serve_groups: int = 0  # serving: traversal groups, each on its own stream (0 = 1)
    stream: int = 0

    def to_c(self) -> N.CgpOptions:
        o = N.default_options()
        if self.traversal_mode not in MODES:
            raise ValueError("traversal_mode must be push, pull, or hybrid")
        o.traversal_mode = MODES[self.traversal_mode]
        o.pull_frontier_ratio = self.pull_frontier_ratio
        o.pull_edge_ratio = self.pull_edge_ratio
        o.profile_iterations = int(self.profile_iterations)
        o.max_iterations = self.max_iterations
        o.max_queries = self.max_queries
        o.discard_results = int(self.discard_results)
        o.use_cuda_graph = int(self.use_cuda_graph)
        o.levels_per_sync = self.levels_per_sync
        o.mask_words = self.mask_words
        o.depth_mode = {"auto": N.DEPTH_AUTO, "planes": N.DEPTH_PLANES,
                        "direct": N.DEPTH_DIRECT}[self.depth_mode]
        o.heavy_degree = self.heavy_degree
        o.profile_kernels = int(self.profile_kernels)
        o.dense_unroll = self.dense_unroll
        o.sssp_pull_edge_ratio = self.sssp_pull_edge_ratio
        o.sssp_pull_pair_ratio = self.sssp_pull_pair_ratio
        o.light_chunks = 0 if self.light_chunks else -1
        if self.level_loop not in ("auto", "chunks", "device"):
            raise ValueError("level_loop must be auto, chunks or device")
        o.level_loop = {"auto": N.LOOP_AUTO, "chunks": N.LOOP_CHUNKS,
                        "device": N.LOOP_DEVICE}[self.level_loop]
        o.sssp_chunk_direction = int(self.sssp_chunk_direction)
        if self.bfs_pull_form not in (0, 1, 2):
            raise ValueError("bfs_pull_form must be 0, 1 or 2")
        o.bfs_pull_form = 1 if self.bfs_pull_chunks else int(self.bfs_pull_form)
        if self.serve_admission not in ("slots", "chunks", "group"):
            raise ValueError("serve_admission must be slots, chunks or group")
        o.serve_admission = {"slots": 0, "chunks": 1, "group": 2}[self.serve_admission]
        if not 0 <= self.serve_groups <= 8:
            raise ValueError("serve_groups must be in [0, 8]")
        o.serve_groups = int(self.serve_groups)
        o.stream = self.stream or None
        return o


@dataclass
class IterationProfile:
    """iteration_profile_t (core/result.hxx:21-46), device-recorded fields."""
    iteration: int
    mode: str
    frontier_size: int
    frontier_edges: int
    next_size: int
    query_convergence_mask: int
    new_pairs: int = 0
    pull_vertices: int = 0
    pull_edges: int = 0
    sssp_pairs: int = 0
    sssp_active: int = 0
    improved: int = 0
    sssp_pull_vertices: int = 0
    sssp_pull_edges: int = 0
    sssp_mode: str = "push"
    kernel_ms: float = 0.0


@dataclass
class RunResult:
    """run_result_t (core/result.hxx:49-66)."""
    values: object
    iterations: int
    gpu_time_ms: float
    wall_time_ms: float
    push_levels: int = 0
    pull_levels: int = 0
    groups: int = 0
    frontier_vertices: int = 0
    frontier_edges: int = 0
    mask_words: int = 0
    depth_mode: str = ""
    effective_query_dim: int = 0
    kernel_launches: int = 0
    counters: dict = field(default_factory=dict)
    kernel_profile: dict = field(default_factory=dict)
    iteration_profiles: list = field(default_factory=list)
    options: RunOptions | None = None


def _queries_c(descs: Sequence[QueryDescriptor]):
    arr = (N.CgpQuery * len(descs))()
    for i, d in enumerate(descs):
        if d.kind not in POLICIES:
            raise ValueError(f"unknown query kind {d.kind!r}")
        arr[i].source = int(d.source)
        arr[i].kind = POLICIES[d.kind]
        arr[i].k = int(d.k)
    return arr


def _dtype_for(kind: str, graph: CsrGraph):
    if kind in ("bfs", "khop"):
        return np.int32
    if kind == "sssp":
        return np.float32 if graph.weight_kind == N.WEIGHT_F32 else np.uint32
    return np.uint32


def run_batch(graph: CsrGraph, descs: Sequence[QueryDescriptor], options: RunOptions | None = None,
              layout: str = "vertex", out=None) -> RunResult:
    """Runs a batch through cgp_batch_run.  `out` may be a device buffer
    (anything with .data_ptr() and .is_cuda, e.g. a torch tensor) or None
    (a host numpy array is returned)."""
    options = options or RunOptions()
    descs = list(descs)
    if not descs:
        raise ValueError("query batch must be non-empty")
    q = _queries_c(descs)
    o = options.to_c()
    V = graph.num_vertices
    lay = N.LAYOUT_QUERY_MAJOR if layout == "query" else N.LAYOUT_VERTEX_MAJOR
    stats = N.CgpStats()
    on_dev = 0
    if out is None:
        kinds = {d.kind for d in descs}
        dt = _dtype_for(descs[0].kind, graph) if len(kinds) == 1 else np.uint32
        arr = np.empty((len(descs), V) if lay == N.LAYOUT_QUERY_MAJOR else (V, len(descs)), dt)
        ptr = arr.ctypes.data
    else:
        arr = out
        ptr = out.data_ptr()
        on_dev = 1 if getattr(out, "is_cuda", False) else 0
    N.check(N.lib().cgp_batch_run(graph.handle, q, len(descs), ctypes.byref(o), ptr, lay, on_dev,
                                  ctypes.byref(stats)), "cgp_batch_run")
    profiles = []
    if options.profile_iterations:
        cnt = ctypes.c_int32()
        N.lib().cgp_last_profiles(None, 0, ctypes.byref(cnt))
        buf = (N.CgpLevelProfile * max(cnt.value, 1))()
        N.lib().cgp_last_profiles(buf, cnt.value, ctypes.byref(cnt))
        profiles = [IterationProfile(p.iteration, "pull" if p.mode else "push", p.frontier_size,
                                     p.frontier_edges, p.next_size, p.query_convergence_mask,
                                     p.new_pairs, p.pull_vertices, p.pull_edges, p.sssp_pairs,
                                     p.sssp_active, p.improved, p.sssp_pull_vertices,
                                     p.sssp_pull_edges, "pull" if p.sssp_mode else "push",
                                     p.kernel_ms)
                    for p in buf[:cnt.value]]
    kprof = {}
    if options.profile_kernels:
        kp = N.CgpKernelProfile()
        N.check(N.lib().cgp_last_kernel_profile(ctypes.byref(kp)))
        kprof = {name: (kp.ms[i], kp.launches[i]) for i, name in enumerate(N.KERNEL_CLASSES)
                 if name and kp.launches[i]}
    return RunResult(values=arr, iterations=stats.iterations, gpu_time_ms=stats.gpu_time_ms,
                     wall_time_ms=stats.wall_time_ms, push_levels=stats.push_levels,
                     pull_levels=stats.pull_levels, groups=stats.groups,
                     frontier_vertices=stats.frontier_vertices,
                     frontier_edges=stats.frontier_edges, mask_words=stats.mask_words,
                     depth_mode="planes" if stats.depth_mode == N.DEPTH_PLANES else "direct",
                     effective_query_dim=len(descs), kernel_launches=stats.kernel_launches,
                     counters={k: getattr(stats, k) for k in ("new_pairs", "pull_vertices",
                                                              "pull_edges", "sssp_pairs",
                                                              "sssp_active", "improved",
                                                              "sssp_pull_vertices",
                                                              "sssp_pull_edges")},
                     kernel_profile=kprof, iteration_profiles=profiles, options=options)


def autotune(graph: CsrGraph, descs: Sequence[QueryDescriptor], options: RunOptions | None = None,
             reps: int = 3) -> RunOptions:
    """Times short runs of `descs` and returns options with the fastest mask
    width, heavy-vertex threshold and pull threshold (cached per graph and
    query mix)."""
    options = options or RunOptions()
    o = options.to_c()
    q = _queries_c(list(descs))
    N.check(N.lib().cgp_autotune(graph.handle, q, len(descs), ctypes.byref(o), reps), "cgp_autotune")
    return dataclasses.replace(options, mask_words=o.mask_words, heavy_degree=o.heavy_degree,
                               pull_edge_ratio=o.pull_edge_ratio,
                               pull_frontier_ratio=o.pull_frontier_ratio,
                               dense_unroll=o.dense_unroll,
                               sssp_pull_edge_ratio=o.sssp_pull_edge_ratio,
                               light_chunks=o.light_chunks >= 0)


def run(policy: str, graph: CsrGraph, queries, context=None, options: RunOptions | None = None,
        **kw) -> RunResult:
    """puercgp::run<Policy> (run.hxx:11-23): one policy over a batch of sources.
    Results are vertex-major values[v*Q + q] like frontier_engine.hxx:3137."""
    if policy not in POLICIES:
        raise ValueError(f"unknown policy {policy!r}")
    qb = queries if isinstance(queries, QueryBatch) else QueryBatch(queries)
    options = options or RunOptions()
    qb.validate(options.max_queries)
    descs = [QueryDescriptor(s, policy) for s in qb.sources]
    return run_batch(graph, descs, options, **kw)


def run_heterogeneous(graph: CsrGraph, batch: HybridQueryBatch, context=None,
                      options: RunOptions | None = None, **kw) -> RunResult:
    """run_heterogeneous (hybrid_engine.hxx:1144-1150): BFS, SSSP, k-hop and
    WCC slots in one traversal.  Values are 4-byte words per (vertex, slot):
    int32 depths, uint32/f32 distances, uint32 labels (view with .view())."""
    options = options or RunOptions()
    batch.validate(options.max_queries)
    return run_batch(graph, batch.descs, options, **kw)


# ---------------------------------------------------------------- operators
class Enactor:
    """Gunrock problem/enactor over one group of <= 1024 queries
    (problem.hxx:28-58, enactor.hxx:78-344)."""

    def __init__(self, graph: CsrGraph, descs: Sequence[QueryDescriptor],
                 options: RunOptions | None = None):
        self.graph = graph
        self.descs = list(descs)
        self.options = options or RunOptions()
        q = _queries_c(self.descs)
        o = self.options.to_c()
        h = ctypes.c_void_p()
        N.check(N.lib().cgp_enactor_create(graph.handle, q, len(self.descs), ctypes.byref(o),
                                           ctypes.byref(h)), "cgp_enactor_create")
        self._h = h
        self.iteration = 0

    def prepare_frontier(self) -> None:
        N.check(N.lib().cgp_enactor_prepare_frontier(self._h), "prepare_frontier")
        self.iteration = 0

    reset = prepare_frontier

    def loop(self, direction: str = "hybrid") -> int:
        """One fused advance+filter level; returns the next frontier size."""
        n = ctypes.c_int64()
        N.check(N.lib().cgp_advance_filter_level(self._h, MODES[direction], ctypes.byref(n)),
                "advance_filter_level")
        self.iteration += 1
        return n.value

    advance_filter = loop

    def is_converged(self) -> bool:
        c = ctypes.c_int32()
        N.check(N.lib().cgp_enactor_is_converged(self._h, ctypes.byref(c)), "is_converged")
        return bool(c.value)

    def enact(self) -> N.CgpStats:
        s = N.CgpStats()
        N.check(N.lib().cgp_enactor_enact(self._h, ctypes.byref(s)), "enact")
        return s

    def frontier(self):
        """(vertex ids, masks[n, mask_words]) of the current frontier."""
        n, w = ctypes.c_int64(), ctypes.c_int32()
        N.check(N.lib().cgp_enactor_frontier(self._h, None, None, 0, ctypes.byref(n),
                                             ctypes.byref(w)))
        vs = np.zeros(n.value, np.int32)
        ms = np.zeros((n.value, w.value), np.uint64)
        if n.value:
            N.check(N.lib().cgp_enactor_frontier(self._h, vs.ctypes.data, ms.ctypes.data, n.value,
                                                 ctypes.byref(n), ctypes.byref(w)))
        return vs, ms

    def values(self, layout: str = "vertex") -> np.ndarray:
        V = self.graph.num_vertices
        q = len(self.descs)
        lay = N.LAYOUT_QUERY_MAJOR if layout == "query" else N.LAYOUT_VERTEX_MAJOR
        arr = np.empty((q, V) if lay else (V, q), np.uint32)
        N.check(N.lib().cgp_enactor_read_values(self._h, arr.ctypes.data, lay, 0), "read_values")
        return arr

    def close(self):
        if getattr(self, "_h", None):
            N.lib().cgp_enactor_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ serving
STATE_NAMES = {0: "queued", 1: "running", 2: "done", 3: "cancelled", 4: "failed"}


@dataclass
class RequestInfo:
    """Per-request record (query_result_t, core/result.hxx:13-19, plus times)."""
    ticket: int
    state: str
    slot: int
    admit_level: int
    completion_level: int
    submit_ms: float
    admit_ms: float
    finish_ms: float

    @property
    def latency_ms(self) -> float:
        return self.finish_ms - self.submit_ms


class Server:
    """Continuous-batching query server (replenish_frontier_engine,
    replenish_engine.hxx:42-554): requests are admitted into free bitmask
    slots at level boundaries while others run; results land in the buffer
    given at submit time."""

    def __init__(self, graph: CsrGraph, slots: int = 64, options: RunOptions | None = None,
                 max_state_bytes: int = 0):
        self.graph = graph
        o = (options or RunOptions()).to_c()
        h = ctypes.c_void_p()
        N.check(N.lib().cgp_server_create(graph.handle, slots, ctypes.byref(o), max_state_bytes,
                                          ctypes.byref(h)), "cgp_server_create")
        self._h = h
        self._keep = {}

    def submit(self, desc: QueryDescriptor, out=None) -> int:
        """Queues a request; `out` is a host numpy array / pinned tensor or a
        device tensor of V 4-byte values, or None (result discarded)."""
        q = _queries_c([desc])
        t = ctypes.c_uint64()
        ptr, on_dev = None, 0
        if out is not None:
            if hasattr(out, "data_ptr"):
                ptr, on_dev = out.data_ptr(), int(bool(getattr(out, "is_cuda", False)))
            else:
                ptr = out.ctypes.data
        N.check(N.lib().cgp_server_submit(self._h, q, ptr, on_dev, ctypes.byref(t)), "submit")
        if out is not None:
            self._keep[t.value] = out
        return t.value

    def _info(self, t, i) -> RequestInfo:
        return RequestInfo(t, STATE_NAMES.get(i.state, "?"), i.slot, i.admit_level,
                           i.completion_level, i.submit_time_ms, i.admit_time_ms,
                           i.finish_time_ms)

    def poll(self, ticket: int) -> RequestInfo:
        i = N.CgpRequestInfo()
        N.check(N.lib().cgp_server_poll(self._h, ticket, ctypes.byref(i)), "poll")
        return self._info(ticket, i)

    def wait(self, ticket: int, timeout_ms: int = -1) -> RequestInfo:
        i = N.CgpRequestInfo()
        N.check(N.lib().cgp_server_wait(self._h, ticket, timeout_ms, ctypes.byref(i)), "wait")
        self._keep.pop(ticket, None)
        return self._info(ticket, i)

    def cancel(self, ticket: int) -> None:
        N.check(N.lib().cgp_server_cancel(self._h, ticket), "cancel")

    def drain(self, timeout_ms: int = -1) -> None:
        N.check(N.lib().cgp_server_drain(self._h, timeout_ms), "drain")

    def stats(self) -> dict:
        s = N.CgpServerStats()
        N.check(N.lib().cgp_server_get_stats(self._h, ctypes.byref(s)), "stats")
        d = {k: getattr(s, k) for k, _ in N.CgpServerStats._fields_ if k != "kernel_ms"}
        d["kernel_ms"] = {name: s.kernel_ms[i] for i, name in enumerate(N.KERNEL_CLASSES)
                          if name and s.kernel_ms[i] > 0}
        return d

    def close(self):
        if getattr(self, "_h", None):
            N.lib().cgp_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_replenish_pipeline(graph: CsrGraph, queries: Sequence[QueryDescriptor], context=None,
                           options: RunOptions | None = None, slots: int = 64) -> RunResult:
    """run_replenish_pipeline (replenish_engine.hxx:559-573): all N queries
    through `slots` bitmask slots, slots reused as queries converge.  Values
    are row-major [N][V] like the reference's final buffer; queries carries
    one RequestInfo per query (completion level and wall time)."""
    options = options or RunOptions()
    queries = list(queries)
    if not queries:
        raise ValueError("replenish: query list must be non-empty")
    if not options.enable_replenishment:
        if len(queries) > 1024:
            raise ValueError("enable_replenishment=false but query count > 1024")
        return run_heterogeneous(graph, HybridQueryBatch(queries), options=options, layout="query")
    V = graph.num_vertices
    vals = np.empty((len(queries), V), np.uint32)
    t0 = __import__("time").perf_counter()
    with Server(graph, min(slots, len(queries)), options) as s:
        tickets = [s.submit(q, None if options.discard_results else vals[i])
                   for i, q in enumerate(queries)]
        s.drain()
        infos = [s.wait(t) for t in tickets]
    wall = (__import__("time").perf_counter() - t0) * 1e3
    res = RunResult(values=vals, iterations=max(i.admit_level + i.completion_level for i in infos),
                    gpu_time_ms=0.0, wall_time_ms=wall, effective_query_dim=len(queries),
                    options=options)
    res.queries = infos
    return res
