"""ctypes view of the C ABI declared in include/cgp_b200.h.

Loading fails loudly when the native library has not been built: there is no
Python or CPU fallback for any traversal.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int32, c_int64,
                    c_size_t, c_uint8, c_uint64, c_void_p)
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcgp_b200.so"

# status codes (cgp_status)
OK, ERR_INVALID_ARG, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_CANCELLED, ERR_NOT_FOUND, \
    ERR_BUSY, ERR_DEVICE = range(9)
KIND_BFS, KIND_SSSP, KIND_WCC, KIND_KHOP = range(4)
MODE_PUSH, MODE_PULL, MODE_HYBRID = range(3)
WEIGHT_NONE, WEIGHT_U32, WEIGHT_F32 = range(3)
LAYOUT_VERTEX_MAJOR, LAYOUT_QUERY_MAJOR = range(2)
DEPTH_AUTO, DEPTH_PLANES, DEPTH_DIRECT = range(3)
LOOP_AUTO, LOOP_CHUNKS, LOOP_DEVICE = range(3)
GRAPH_DEVICE_POINTERS, GRAPH_SYMMETRIC, GRAPH_OFFSETS64 = 1, 2, 4
BFS_UNREACHED = 2**31 - 1
U32_UNREACHED = 2**32 - 1


class CgpQuery(Structure):
    _fields_ = [("source", c_int32), ("kind", c_int32), ("k", c_int32), ("reserved", c_int32)]


class CgpOptions(Structure):
    _fields_ = [
        ("traversal_mode", c_int32), ("push_strategy", c_int32), ("pull_strategy", c_int32),
        ("max_iterations", c_int32), ("pull_frontier_ratio", c_double),
        ("pull_edge_ratio", c_double), ("profile_iterations", c_int32),
        ("use_cuda_graph", c_int32), ("levels_per_sync", c_int32), ("mask_words", c_int32),
        ("depth_mode", c_int32), ("heavy_degree", c_int32), ("max_queries", c_int32),
        ("discard_results", c_int32), ("profile_kernels", c_int32), ("dense_unroll", c_int32),
        ("sssp_pull_edge_ratio", c_double), ("light_chunks", c_int32), ("level_loop", c_int32),
        ("sssp_chunk_direction", c_int32), ("bfs_pull_form", c_int32),
        ("serve_admission", c_int32), ("serve_groups", c_int32),
        ("sssp_pull_pair_ratio", c_double), ("stream", c_void_p),
    ]


class CgpLevelProfile(Structure):
    _fields_ = [("iteration", c_int32), ("mode", c_int32), ("frontier_size", c_uint64),
                ("frontier_edges", c_uint64), ("next_size", c_uint64),
                ("query_convergence_mask", c_uint64), ("new_pairs", c_uint64),
                ("pull_vertices", c_uint64), ("pull_edges", c_uint64), ("sssp_pairs", c_uint64),
                ("sssp_active", c_uint64), ("improved", c_uint64),
                ("sssp_pull_vertices", c_uint64), ("sssp_pull_edges", c_uint64),
                ("sssp_mode", c_int32), ("kernel_ms", c_float)]


class CgpStats(Structure):
    _fields_ = [("iterations", c_int32), ("push_levels", c_int32), ("pull_levels", c_int32),
                ("groups", c_int32), ("gpu_time_ms", c_float), ("wall_time_ms", c_float),
                ("frontier_vertices", c_uint64), ("frontier_edges", c_uint64),
                ("device_status", c_uint64), ("mask_words", c_int32), ("depth_mode", c_int32),
                ("kernel_launches", c_uint64), ("new_pairs", c_uint64), ("pull_vertices", c_uint64),
                ("pull_edges", c_uint64), ("sssp_pairs", c_uint64), ("sssp_active", c_uint64),
                ("improved", c_uint64), ("sssp_pull_vertices", c_uint64),
                ("sssp_pull_edges", c_uint64)]


KERNEL_CLASSES = ["clear", "bfs_push", "bfs_pull", "sssp_push", "level_end", "init", "output",
                  "wcc", "sssp_dense", "sssp_heavy", "sssp_pull", ""]


class CgpKernelProfile(Structure):
    _fields_ = [("ms", c_double * 12), ("launches", c_int64 * 12)]


class CgpHostCsr(Structure):
    _fields_ = [("num_vertices", c_int64), ("num_edges", c_int64),
                ("row_offsets", POINTER(c_int64)), ("col_indices", POINTER(c_int32)),
                ("weights", c_void_p), ("weight_kind", c_int32), ("reserved", c_int32)]


class CgpRequestInfo(Structure):
    _fields_ = [("state", c_int32), ("slot", c_int32), ("admit_level", c_int32),
                ("completion_level", c_int32), ("submit_time_ms", c_double),
                ("admit_time_ms", c_double), ("finish_time_ms", c_double)]


class CgpServerStats(Structure):
    _fields_ = [("slots", c_int32), ("active_slots", c_int32), ("queued", c_int64),
                ("completed", c_int64), ("levels", c_int64), ("busy_ms", c_double),
                ("state_bytes", c_int64), ("admit_ms", c_double), ("retire_ms", c_double),
                ("retire_passes", c_int64), ("kernel_ms", c_double * 12),
                ("sssp_chunk_levels", c_int64), ("gather_chunk_levels", c_int64)]


# name -> (restype, argtypes)
SIGNATURES = {
    "cgp_last_error": (c_int32, [c_char_p, c_size_t]),
    "cgp_status_name": (c_char_p, [c_int32]),
    "cgp_options_init": (c_int32, [POINTER(CgpOptions)]),
    "cgp_version": (c_char_p, []),
    "cgp_set_device": (c_int32, [c_int32]),
    "cgp_last_kernel_profile": (c_int32, [POINTER(CgpKernelProfile)]),
    "cgp_debug_fail_allocations": (c_int32, [c_int64]),
    "cgp_graph_create": (c_int32, [c_void_p, c_int32, c_void_p, c_void_p, c_int32, c_int64,
                                   c_int64, c_int32, POINTER(c_void_p)]),
    "cgp_graph_destroy": (c_int32, [c_void_p]),
    "cgp_graph_info": (c_int32, [c_void_p, POINTER(c_int64), POINTER(c_int64),
                                 POINTER(c_int32), POINTER(c_int32)]),
    "cgp_batch_run": (c_int32, [c_void_p, POINTER(CgpQuery), c_int32, POINTER(CgpOptions),
                                c_void_p, c_int32, c_int32, POINTER(CgpStats)]),
    "cgp_last_profiles": (c_int32, [POINTER(CgpLevelProfile), c_int32, POINTER(c_int32)]),
    "cgp_autotune": (c_int32, [c_void_p, POINTER(CgpQuery), c_int32, POINTER(CgpOptions), c_int32]),
    "cgp_enactor_create": (c_int32, [c_void_p, POINTER(CgpQuery), c_int32, POINTER(CgpOptions),
                                     POINTER(c_void_p)]),
    "cgp_enactor_destroy": (c_int32, [c_void_p]),
    "cgp_enactor_prepare_frontier": (c_int32, [c_void_p]),
    "cgp_advance_filter_level": (c_int32, [c_void_p, c_int32, POINTER(c_int64)]),
    "cgp_enactor_is_converged": (c_int32, [c_void_p, POINTER(c_int32)]),
    "cgp_enactor_enact": (c_int32, [c_void_p, POINTER(CgpStats)]),
    "cgp_enactor_frontier": (c_int32, [c_void_p, c_void_p, c_void_p, c_int64, POINTER(c_int64),
                                       POINTER(c_int32)]),
    "cgp_enactor_read_values": (c_int32, [c_void_p, c_void_p, c_int32, c_int32]),
    "cgp_gen_rmat": (c_int32, [c_int32, c_int32, c_double, c_double, c_double, c_uint64, c_int32,
                               POINTER(CgpHostCsr)]),
    "cgp_gen_grid": (c_int32, [c_int32, c_int32, c_double, c_double, c_uint64,
                               POINTER(CgpHostCsr)]),
    "cgp_gen_chung_lu": (c_int32, [c_int64, c_double, c_double, c_uint64, POINTER(CgpHostCsr)]),
    "cgp_gen_weights": (c_int32, [POINTER(CgpHostCsr), c_int32, c_double, c_double, c_int32,
                                  c_uint64]),
    "cgp_csr_from_edges": (c_int32, [c_int64, c_int64, c_void_p, c_void_p, c_int32,
                                     POINTER(CgpHostCsr)]),
    "cgp_pick_sources": (c_int32, [POINTER(CgpHostCsr), c_int32, c_int32, c_void_p, c_uint64,
                                   c_void_p]),
    "cgp_load_matrix_market": (c_int32, [c_char_p, POINTER(CgpHostCsr)]),
    "cgp_load_binary_csr": (c_int32, [c_char_p, POINTER(CgpHostCsr)]),
    "cgp_load_galois_gr": (c_int32, [c_char_p, c_int32, POINTER(CgpHostCsr)]),
    "cgp_host_csr_free": (None, [POINTER(CgpHostCsr)]),
}

OPTIONAL = {
    "cgp_server_create": (c_int32, [c_void_p, c_int32, POINTER(CgpOptions), c_int64,
                                    POINTER(c_void_p)]),
    "cgp_server_destroy": (c_int32, [c_void_p]),
    "cgp_server_submit": (c_int32, [c_void_p, POINTER(CgpQuery), c_void_p, c_int32,
                                    POINTER(c_uint64)]),
    "cgp_server_poll": (c_int32, [c_void_p, c_uint64, POINTER(CgpRequestInfo)]),
    "cgp_server_wait": (c_int32, [c_void_p, c_uint64, c_int32, POINTER(CgpRequestInfo)]),
    "cgp_server_cancel": (c_int32, [c_void_p, c_uint64]),
    "cgp_server_drain": (c_int32, [c_void_p, c_int32]),
    "cgp_server_get_stats": (c_int32, [c_void_p, POINTER(CgpServerStats)]),
}

_lib = None


def lib():
    """The loaded native library (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"native library {LIB_PATH} is missing; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` or "
                "`python cgp_b200/build.py`")
        l = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in {**SIGNATURES, **OPTIONAL}.items():
            if not hasattr(l, name):
                if name in SIGNATURES:
                    raise ImportError(f"{LIB_PATH} does not export {name}")
                continue
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


class CgpError(RuntimeError):
    """Native call failed; `status` holds the cgp_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class CgpInvalidArgument(CgpError, ValueError):
    """CGP_ERR_INVALID_ARG: the reference raises std::invalid_argument here."""


class CgpOutOfMemory(CgpError, MemoryError):
    """CGP_ERR_OOM."""


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    lib().cgp_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, what: str = "") -> None:
    if status == OK:
        return
    name = lib().cgp_status_name(status).decode()
    msg = f"{what}: {name}: {last_error()}" if what else f"{name}: {last_error()}"
    if status == ERR_INVALID_ARG:
        raise CgpInvalidArgument(status, msg)
    if status == ERR_OOM:
        raise CgpOutOfMemory(status, msg)
    raise CgpError(status, msg)


def default_options() -> CgpOptions:
    o = CgpOptions()
    check(lib().cgp_options_init(ctypes.byref(o)), "cgp_options_init")
    return o


def declared_symbols(header: os.PathLike | None = None) -> list[str]:
    """Function names declared in include/cgp_b200.h."""
    import re
    h = Path(header) if header else Path(__file__).resolve().parent.parent / "include" / "cgp_b200.h"
    text = h.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cgp_[a-z0-9_]+)\s*\(", text)))
