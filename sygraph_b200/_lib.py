"""ctypes binding of libsygraph_b200.so (declarations of include/sygraph_b200.h).

The library is required: importing this module without a built
``libsygraph_b200.so`` raises ImportError.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsygraph_b200.so"

SG_OK = 0
SG_ERR_INVALID = 1
SG_ERR_CUDA = 2
SG_ERR_NOMEM = 3
SG_ERR_TIMEOUT = 4
SG_ERR_UNSUPPORTED = 5
SG_ERR_NOT_INITIALIZED = 6

SG_MAX_LOGGED_LEVELS = 4096

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
i32p = C.POINTER(C.c_int32)
f32p = C.POINTER(C.c_float)
vp = C.c_void_p
st = C.c_int


class GraphView(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("row_offsets", u32p), ("column_indices", u32p),
                ("values", vp), ("value_type", C.c_int)]


class FrontierView(C.Structure):
    _fields_ = [("num_elems", C.c_uint32), ("words0", C.c_uint32), ("words1", C.c_uint32), ("level0", u32p),
                ("level1", u32p), ("offsets", i32p), ("offsets_size", u32p)]


class OpArgs(C.Structure):
    _fields_ = [("p", vp * 4), ("u", C.c_uint32 * 4), ("f", C.c_float * 4)]


class BfsDetails(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("push_steps", C.c_uint64), ("pull_steps", C.c_uint64),
                ("visited_vertices", C.c_uint64), ("visited_edges", C.c_uint64),
                ("step_is_pull", C.c_uint8 * SG_MAX_LOGGED_LEVELS)]


class LevelRecord(C.Structure):
    _fields_ = [("level", C.c_uint32), ("strategy", C.c_uint32), ("frontier_size", C.c_uint32),
                ("next_size", C.c_uint32), ("frontier_degree", C.c_uint64), ("next_degree", C.c_uint64),
                ("unexplored_degree", C.c_uint64), ("t_start_ns", C.c_uint64), ("t_end_ns", C.c_uint64)]


class MsbfsDetails(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("push_steps", C.c_uint64), ("pull_steps", C.c_uint64),
                ("reached_edges", C.c_uint64)]


class BcBatchDetails(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("reached_edges", C.c_uint64), ("history_levels", C.c_uint64),
                ("history_retries", C.c_uint64)]


class ServerConfig(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("max_batch", C.c_uint32), ("min_batch", C.c_uint32),
                ("ctas_per_slot", C.c_uint32), ("memory_budget", C.c_uint64), ("sssp_delta", C.c_double)]


class QueryResult(C.Structure):
    _fields_ = [("status", C.c_int), ("graph", C.c_uint32), ("source", C.c_uint32), ("batch_size", C.c_uint32),
                ("kind", C.c_int), ("submit_ns", C.c_uint64), ("start_ns", C.c_uint64), ("end_ns", C.c_uint64)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "failed", "launches", "batched_queries",
                                          "evictions", "deferred_admissions", "workspace_bytes",
                                          "peak_workspace_bytes", "memory_budget")]


class HostCSR(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("row_offsets", u32p), ("column_indices", u32p),
                ("values", vp), ("value_type", C.c_int), ("flags", C.c_uint32)]


class RmatParams(C.Structure):
    _fields_ = [("scale", C.c_uint32), ("edge_factor", C.c_uint32), ("a", C.c_double), ("b", C.c_double),
                ("c", C.c_double), ("seed", C.c_uint64), ("weight_seed", C.c_uint64), ("perm_seed", C.c_uint64),
                ("value_type", C.c_int)]


# name -> (restype, argtypes)
SIGNATURES = {
    "sg_last_error": (C.c_char_p, []),
    "sg_status_string": (C.c_char_p, [st]),
    "sg_version": (C.c_char_p, []),
    "sg_kernel_launch_count": (C.c_uint64, []),
    "sg_device_count": (st, [C.POINTER(C.c_int)]),
    "sg_set_device": (st, [C.c_int]),
    "sg_device_info": (st, [C.POINTER(C.c_int), u64p, u64p]),
    "sg_malloc_device": (st, [C.c_uint64, C.POINTER(vp)]),
    "sg_free_device": (st, [vp]),
    "sg_malloc_host_pinned": (st, [C.c_uint64, C.POINTER(vp)]),
    "sg_free_host_pinned": (st, [vp]),
    "sg_memcpy": (st, [vp, vp, C.c_uint64, C.c_int, vp]),
    "sg_memcpy_async": (st, [vp, vp, C.c_uint64, C.c_int, vp]),
    "sg_memset": (st, [vp, C.c_int, C.c_uint64, vp]),
    "sg_debug_barrier_check": (st, [C.c_uint32, C.c_uint32, C.c_uint64, u32p, u32p]),
    "sg_event_record": (st, [vp, C.POINTER(vp)]),
    "sg_event_elapsed_ms": (st, [vp, vp, C.POINTER(C.c_float)]),
    "sg_event_destroy": (st, [vp]),
    "sg_stream_create": (st, [C.POINTER(vp)]),
    "sg_stream_destroy": (st, [vp]),
    "sg_stream_synchronize": (st, [vp]),
    "sg_device_synchronize": (st, []),
    # graph
    "sg_graph_create_csr": (st, [u32p, u32p, vp, C.c_int, C.c_uint32, C.c_uint64, C.c_uint32, vp, C.POINTER(vp)]),
    "sg_graph_create_coo": (st, [vp, vp, vp, C.c_int, C.c_uint32, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, vp,
                                 C.POINTER(vp)]),
    "sg_graph_destroy": (st, [vp]),
    "sg_graph_info": (st, [vp, u32p, u64p, u32p, C.POINTER(C.c_int)]),
    "sg_graph_device_view": (st, [vp, C.c_int, C.POINTER(GraphView)]),
    "sg_graph_set_stream": (st, [vp, vp]),
    "sg_graph_copy_csr": (st, [vp, C.c_int, u32p, u32p, vp]),
    "sg_graph_degree": (st, [vp, C.c_uint32, u32p]),
    "sg_graph_memory_bytes": (st, [vp, u64p]),
    "sg_graph_weight_sorted": (st, [vp, u32p, vp, C.POINTER(C.c_int)]),
    # frontier
    "sg_frontier_create": (st, [C.c_uint32, vp, C.POINTER(vp)]),
    "sg_frontier_destroy": (st, [vp]),
    "sg_frontier_device_view": (st, [vp, C.POINTER(FrontierView)]),
    "sg_frontier_num_elems": (st, [vp, u32p]),
    "sg_frontier_clear": (st, [vp]),
    "sg_frontier_insert": (st, [vp, C.c_uint32]),
    "sg_frontier_remove": (st, [vp, C.c_uint32]),
    "sg_frontier_check": (st, [vp, C.c_uint32, C.POINTER(C.c_int)]),
    "sg_frontier_insert_list": (st, [vp, u32p, C.c_uint64]),
    "sg_frontier_empty": (st, [vp, C.POINTER(C.c_int)]),
    "sg_frontier_size": (st, [vp, u64p]),
    "sg_frontier_merge": (st, [vp, vp]),
    "sg_frontier_intersect": (st, [vp, vp]),
    "sg_frontier_swap": (st, [vp, vp]),
    "sg_frontier_compact": (st, [vp, C.c_int, u32p]),
    "sg_frontier_save": (st, [vp, u32p, u32p]),
    "sg_frontier_load": (st, [vp, u32p, u32p]),
    "sg_frontier_to_flags": (st, [vp, u8p]),
    # operators
    "sg_advance": (st, [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(OpArgs), C.c_int]),
    "sg_filter_external": (st, [vp, vp, vp, C.c_int, C.POINTER(OpArgs)]),
    "sg_filter_inplace": (st, [vp, vp, C.c_int, C.POINTER(OpArgs)]),
    "sg_compute_execute": (st, [vp, vp, C.c_int, C.POINTER(OpArgs)]),
    "sg_compute_reduce": (st, [vp, vp, C.c_int, C.POINTER(OpArgs), u64p]),
    "sg_intersection_execute": (st, [vp, vp, vp, vp]),
    "sg_segmented_intersection": (st, [vp, u32p, u32p, C.c_uint64, u32p]),
    # algorithms
    "sg_bfs_create": (st, [vp, C.POINTER(vp)]),
    "sg_bfs_destroy": (st, [vp]),
    "sg_bfs_init": (st, [vp, C.c_uint32]),
    "sg_bfs_reset": (st, [vp]),
    "sg_bfs_run": (st, [vp, C.c_int, C.c_float, C.c_float, C.POINTER(BfsDetails)]),
    "sg_bfs_run_async": (st, [vp, C.c_int, C.c_float, C.c_float]),
    "sg_bfs_get_distances": (st, [vp, u32p]),
    "sg_bfs_distances_device": (st, [vp, C.POINTER(u32p)]),
    "sg_bfs_level_records": (st, [vp, C.POINTER(LevelRecord), C.c_uint32, u32p]),
    "sg_run_bfs": (st, [vp, C.c_uint32, C.c_int, C.c_float, C.c_float, u32p, C.POINTER(BfsDetails)]),
    "sg_bfs_set_schedule": (st, [vp, C.POINTER(C.c_int), C.c_uint32]),
    "sg_bfs_set_selector": (st, [vp, vp, C.c_uint32]),
    "sg_bfs_set_selector_min_frontier": (st, [vp, C.c_float]),
    "sg_bfs_set_selector_max_frontier": (st, [vp, C.c_float]),
    "sg_bfs_set_selector_margin": (st, [vp, C.c_float]),
    "sg_bfs_set_pull_order": (st, [vp, C.c_uint64]),
    "sg_bfs_set_pull_words": (st, [vp, C.c_uint32]),
    "sg_bfs_set_selector_graph_range": (st, [vp, C.c_float, C.c_float]),
    "sg_bfs_log_features": (st, [vp, C.c_int]),
    "sg_bfs_level_features": (st, [vp, f32p, C.c_uint32, u32p]),
    "sg_mlp_param_count": (C.c_uint32, []),
    "sg_mlp_create": (st, [f32p, C.POINTER(vp)]),
    "sg_mlp_destroy": (st, [vp]),
    "sg_mlp_get_params": (st, [vp, f32p]),
    "sg_mlp_set_params": (st, [vp, f32p]),
    "sg_mlp_forward": (st, [vp, vp, C.c_uint32, vp]),
    "sg_mlp_gradient": (st, [vp, vp, vp, vp, C.c_uint32, f32p, f32p]),
    "sg_mlp_train": (st, [vp, vp, vp, vp, C.c_uint32, C.c_uint32, C.c_float, C.c_float, f32p]),
    "sg_msbfs_create": (st, [vp, C.c_uint32, C.POINTER(vp)]),
    "sg_server_create": (st, [C.POINTER(ServerConfig), C.POINTER(vp)]),
    "sg_server_destroy": (st, [vp]),
    "sg_server_add_graph": (st, [vp, vp, u32p]),
    "sg_server_prepare": (st, [vp, C.c_uint32]),
    "sg_server_submit": (st, [vp, C.c_uint32, C.c_int, C.c_uint32, vp, u64p]),
    "sg_server_wait": (st, [vp, C.c_uint64, C.c_double, C.POINTER(QueryResult)]),
    "sg_server_drain": (st, [vp, C.c_double]),
    "sg_server_get_stats": (st, [vp, C.POINTER(ServerStats)]),
    "sg_sssp_set_delta": (st, [vp, C.c_double]),
    "sg_sssp_set_tail": (st, [vp, C.c_double]),
    "sg_sssp_set_heavy_pull": (st, [vp, C.c_uint32]),
    "sg_sssp_set_light_pull": (st, [vp, C.c_uint32]),
    "sg_sssp_set_pull": (st, [vp, C.c_uint32]),
    "sg_sssp_level_records": (st, [vp, C.POINTER(LevelRecord), C.c_uint32, u32p]),
    "sg_sssp_set_launch": (st, [vp, vp, C.c_uint32]),
    "sg_bfs_set_launch": (st, [vp, vp, C.c_uint32]),
    "sg_msbfs_set_launch": (st, [vp, vp, C.c_uint32]),
    "sg_bc_batch_create": (st, [vp, C.c_uint32, C.POINTER(vp)]),
    "sg_bc_batch_destroy": (st, [vp]),
    "sg_bc_batch_run_async": (st, [vp, u32p, C.c_uint32, C.c_int]),
    "sg_bc_batch_run": (st, [vp, u32p, C.c_uint32, C.c_int, C.POINTER(BcBatchDetails)]),
    "sg_bc_batch_get": (st, [vp, f32p]),
    "sg_bc_batch_set_launch": (st, [vp, vp, C.c_uint32]),
    "sg_bc_batch_bc_device": (st, [vp, C.POINTER(vp)]),
    "sg_bc_batch_level_records": (st, [vp, C.POINTER(LevelRecord), C.c_uint32, u32p]),
    "sg_bc_batched": (st, [vp, u32p, C.c_uint32, f32p]),
    "sg_msbfs_level_records": (st, [vp, C.POINTER(LevelRecord), C.c_uint32, u32p]),
    "sg_msbfs_set_schedule": (st, [vp, C.POINTER(C.c_int), C.c_uint32]),
    "sg_msbfs_set_selector": (st, [vp, vp, C.c_float, C.c_float, C.c_float]),
    "sg_msbfs_log_features": (st, [vp, C.c_int]),
    "sg_msbfs_level_features": (st, [vp, f32p, C.c_uint32, u32p]),
    "sg_sssp_set_selector": (st, [vp, vp, C.c_float, C.c_float, C.c_float]),
    "sg_sssp_log_features": (st, [vp, C.c_int]),
    "sg_sssp_level_features": (st, [vp, f32p, C.c_uint32, u32p]),
    "sg_msbfs_destroy": (st, [vp]),
    "sg_msbfs_run": (st, [vp, u32p, C.c_uint32, C.c_int, C.c_float, C.c_float, C.POINTER(MsbfsDetails)]),
    "sg_msbfs_run_async": (st, [vp, u32p, C.c_uint32, C.c_int, C.c_float, C.c_float]),
    "sg_msbfs_get_depths": (st, [vp, u32p]),
    "sg_msbfs_depths_device": (st, [vp, C.POINTER(u32p)]),
    "sg_sssp_create": (st, [vp, C.POINTER(vp)]),
    "sg_sssp_destroy": (st, [vp]),
    "sg_sssp_init": (st, [vp, C.c_uint32]),
    "sg_sssp_run": (st, [vp, u64p]),
    "sg_sssp_run_async": (st, [vp]),
    "sg_sssp_get_distances": (st, [vp, vp]),
    "sg_sssp_distances_device": (st, [vp, C.POINTER(vp)]),
    "sg_run_sssp": (st, [vp, C.c_uint32, vp, u64p]),
    "sg_cc": (st, [vp, u32p, u64p]),
    "sg_cc_create": (st, [vp, C.POINTER(vp)]),
    "sg_cc_destroy": (st, [vp]),
    "sg_cc_run_async": (st, [vp]),
    "sg_cc_set_method": (st, [vp, C.c_int]),
    "sg_cc_run": (st, [vp, u64p]),
    "sg_cc_get_labels": (st, [vp, u32p]),
    "sg_cc_labels_device": (st, [vp, C.POINTER(vp)]),
    "sg_bc": (st, [vp, u32p, C.c_uint32, f32p]),
    "sg_tc": (st, [vp, u64p, u64p]),
    "sg_tc_create": (st, [vp, C.POINTER(vp)]),
    "sg_tc_destroy": (st, [vp]),
    "sg_tc_run_async": (st, [vp, C.c_int]),
    "sg_tc_run": (st, [vp, C.c_int, u64p]),
    "sg_tc_get_total": (st, [vp, u64p]),
    "sg_tc_set_shorter_rows": (st, [vp, C.c_int]),
    "sg_tc_get_per_vertex": (st, [vp, u64p]),
    # host graph I/O
    "sg_rmat_generate": (st, [C.POINTER(RmatParams), C.POINTER(HostCSR)]),
    "sg_grid_generate": (st, [C.c_uint32, C.c_double, C.c_uint64, C.c_uint64, C.c_int, C.POINTER(HostCSR)]),
    "sg_csr_from_edges": (st, [C.c_uint32, u32p, u32p, vp, C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_int,
                               C.POINTER(HostCSR)]),
    "sg_csr_invert": (st, [C.POINTER(HostCSR), C.POINTER(HostCSR)]),
    "sg_csr_write_binary": (st, [C.POINTER(HostCSR), C.c_char_p]),
    "sg_csr_read_binary": (st, [C.c_char_p, C.c_int, C.POINTER(HostCSR)]),
    "sg_csr_read_mm": (st, [C.c_char_p, C.c_int, C.POINTER(HostCSR)]),
    "sg_host_csr_free": (None, [C.POINTER(HostCSR)]),
    "sg_sample_sources": (st, [C.POINTER(HostCSR), C.c_uint32, C.c_uint64, u32p]),
}

# Entry points added after the first release; bound when present.
OPTIONAL = {}


class SygraphError(RuntimeError):
    """A C-ABI call returned a status other than SG_OK."""

    def __init__(self, status: int, fn: str, msg: str):
        super().__init__(f"{fn} -> {status}: {msg}")
        self.status = status


MISSING: list[str] = []


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m sygraph_b200.build` (nvcc, sm_100a). "
            "sygraph_b200 has no CPU fallback.")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in {**SIGNATURES, **OPTIONAL}.items():
        fn = getattr(lib, name, None)
        if fn is None:
            MISSING.append(name)
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int, fn: str = "sygraph_b200") -> None:
    if status != SG_OK:
        raise SygraphError(status, fn, lib.sg_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    check(getattr(lib, name)(*args), name)
