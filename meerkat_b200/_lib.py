"""ctypes bindings of libmeerkat_b200.so (the C ABI in include/meerkat_b200.h)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libmeerkat_b200.so"

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)
vp = C.c_void_p

MK_OK, MK_ERR_INVALID, MK_ERR_OOM, MK_ERR_TIMEOUT, MK_ERR_CUDA, MK_ERR_STATE = range(6)
STATUS_NAMES = {0: "MK_OK", 1: "MK_ERR_INVALID", 2: "MK_ERR_OOM", 3: "MK_ERR_TIMEOUT",
                4: "MK_ERR_CUDA", 5: "MK_ERR_STATE"}
MK_INF = 0xFFFFFFFF
# sticky device error bits returned by DynamicGraph.sync() (MK_DEVERR_*)
DEVERR_INVALID_ID, DEVERR_OOM, DEVERR_TIMEOUT, DEVERR_OVERFLOW = 0x1, 0x2, 0x4, 0x8


class GraphDesc(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("weighted", C.c_uint32), ("reverse", C.c_uint32),
                ("flags", C.c_uint32), ("load_factor", C.c_double), ("h_degree_hints", u32p),
                ("device", C.c_int32), ("pad0", C.c_uint32), ("pool_slabs", C.c_uint64)]


class GraphInfo(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("weighted", C.c_uint32), ("reverse", C.c_uint32),
                ("keys_per_slab", C.c_uint32), ("num_buckets", C.c_uint64),
                ("pool_capacity", C.c_uint64), ("slabs_used", C.c_uint64),
                ("num_edges", C.c_uint64), ("device_bytes", C.c_uint64)]


class Tuning(C.Structure):
    _fields_ = [("update_kernel", C.c_uint32), ("update_blocks_per_sm", C.c_uint32),
                ("frontier_chunk", C.c_uint32), ("sssp_delta", C.c_uint32),
                ("recompute_permille", C.c_uint32), ("pull_permille", C.c_uint32),
                ("wait_limit_us", C.c_uint32), ("reserved", C.c_uint32)]


# (name, restype, argtypes); every function returns mk_status unless noted
_S = C.c_int
SIGNATURES = [
    ("mk_last_error_string", C.c_char_p, []),
    ("mk_version", C.c_char_p, []),
    ("mk_graph_create", _S, [C.POINTER(GraphDesc), C.POINTER(vp)]),
    ("mk_graph_destroy", _S, [vp]),
    ("mk_graph_insert_edges", _S, [vp, vp, vp, vp, C.c_uint32, vp]),
    ("mk_graph_delete_edges", _S, [vp, vp, vp, C.c_uint32, vp]),
    ("mk_graph_search_edges", _S, [vp, vp, vp, C.c_uint32, vp, vp, vp]),
    ("mk_graph_sync", _S, [vp, vp, u32p]),
    ("mk_graph_slabs_used_async", _S, [vp, vp, vp]),
    ("mk_graph_last_applied", _S, [vp, u64p]),
    ("mk_graph_last_applied_async", _S, [vp, vp, vp]),
    ("mk_graph_last_applied_flags", _S, [vp, C.POINTER(vp), u32p]),
    ("mk_graph_degrees", _S, [vp, vp, vp]),
    ("mk_graph_bucket_layout", _S, [vp, vp, vp]),
    ("mk_graph_get_info", _S, [vp, C.POINTER(GraphInfo)]),
    ("mk_graph_export_csr", _S, [vp, vp, vp, vp, vp]),
    ("mk_graph_export_csr_noalloc", _S, [vp, vp, vp, vp, vp]),
    ("mk_graph_count_edges_range", _S, [vp, C.c_uint32, C.c_uint32, vp, u64p]),
    ("mk_graph_export_csr_range", _S, [vp, C.c_uint32, C.c_uint32, vp, vp, vp, vp]),
    ("mk_graph_count_tombstones", _S, [vp, vp, vp]),
    ("mk_graph_reserve_batch", _S, [vp, C.c_uint32]),
    ("mk_graph_set_tuning", _S, [vp, C.POINTER(Tuning)]),
    ("mk_graph_get_tuning", _S, [vp, C.POINTER(Tuning)]),
    ("mk_bfs_create", _S, [vp, C.c_uint32, C.POINTER(vp)]),
    ("mk_sssp_create", _S, [vp, C.c_uint32, C.POINTER(vp)]),
    ("mk_bfs_create_multi", _S, [vp, u32p, C.c_uint32, C.POINTER(vp)]),
    ("mk_sssp_create_multi", _S, [vp, u32p, C.c_uint32, C.POINTER(vp)]),
    ("mk_traversal_set_sources", _S, [vp, u32p, C.c_uint32]),
    ("mk_traversal_set_sources_async", _S, [vp, vp, C.c_uint32, vp]),
    ("mk_traversal_set_reverse", _S, [vp, vp]),
    ("mk_traversal_static", _S, [vp, vp, f32p]),
    ("mk_bfs_prepare_members", _S, [vp, u32p, C.c_uint32]),
    ("mk_bfs_static_members", _S, [vp, vp, f32p]),
    ("mk_traversal_incremental", _S, [vp, vp, vp, vp, C.c_uint32, vp, f32p]),
    ("mk_traversal_decremental", _S, [vp, vp, vp, vp, C.c_uint32, vp, f32p]),
    ("mk_traversal_distances", _S, [vp, vp]),
    ("mk_traversal_packed", _S, [vp, C.POINTER(vp)]),
    ("mk_traversal_packed_host", _S, [vp, vp]),
    ("mk_traversal_decremental_stats", _S, [vp, u64p, u32p]),
    ("mk_traversal_stats", _S, [vp, u32p, u64p]),
    ("mk_traversal_destroy", _S, [vp]),
    ("mk_pagerank_create", _S, [vp, C.c_float, C.c_float, C.c_uint32, vp, C.POINTER(vp)]),
    ("mk_pagerank_static", _S, [vp, vp, f32p]),
    ("mk_pagerank_static_recount", _S, [vp, vp, f32p]),
    ("mk_pagerank_incremental", _S, [vp, vp, vp, C.c_uint32, vp, f32p]),
    ("mk_pagerank_decremental", _S, [vp, vp, vp, C.c_uint32, vp, f32p]),
    ("mk_pagerank_values", _S, [vp, vp]),
    ("mk_pagerank_values_device", _S, [vp, C.POINTER(vp)]),
    ("mk_pagerank_stats", _S, [vp, u32p, f32p]),
    ("mk_pagerank_destroy", _S, [vp]),
    ("mk_pagerank_range_create", _S, [vp, C.c_uint32, C.POINTER(vp)]),
    ("mk_pagerank_range_run", _S, [vp, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_uint32,
                                   vp, f32p]),
    ("mk_pagerank_range_values", _S, [vp, vp]),
    ("mk_pagerank_range_stats", _S, [vp, u32p, f32p]),
    ("mk_pagerank_range_destroy", _S, [vp]),
    ("mk_tc_create", _S, [vp, C.POINTER(vp)]),
    ("mk_tc_static", _S, [vp, vp, f32p]),
    ("mk_tc_incremental", _S, [vp, vp, vp, C.c_uint32, vp, f32p]),
    ("mk_tc_decremental", _S, [vp, vp, vp, C.c_uint32, vp, f32p]),
    ("mk_tc_count", _S, [vp, u64p]),
    ("mk_tc_range_create", _S, [vp, C.POINTER(vp)]),
    ("mk_tc_range_run", _S, [vp, C.c_uint32, C.c_uint32, vp, f32p]),
    ("mk_tc_range_count", _S, [vp, u64p]),
    ("mk_tc_range_count_async", _S, [vp, vp, vp]),
    ("mk_tc_range_destroy", _S, [vp]),
    ("mk_tc_destroy", _S, [vp]),
    ("mk_wcc_create", _S, [vp, C.POINTER(vp)]),
    ("mk_wcc_static", _S, [vp, vp, f32p]),
    ("mk_wcc_static_subset", _S, [vp, vp, vp, f32p]),
    ("mk_wcc_static_ranges", _S, [vp, u32p, C.c_uint32, vp, f32p]),
    ("mk_wcc_prepare_ranges", _S, [vp, u32p, C.c_uint32]),
    ("mk_wcc_prepare_ranges_async", _S, [vp, vp, C.c_uint32, vp]),
    ("mk_wcc_static_prepared", _S, [vp, vp, f32p]),
    ("mk_wcc_incremental", _S, [vp, vp, vp, C.c_uint32, vp, f32p]),
    ("mk_wcc_decremental", _S, [vp, vp, vp, C.c_uint32, vp, f32p]),
    ("mk_wcc_set_reverse", _S, [vp, vp]),
    ("mk_wcc_decremental_stats", _S, [vp, u64p, u64p, u32p]),
    ("mk_wcc_labels", _S, [vp, vp]),
    ("mk_wcc_labels_device", _S, [vp, C.POINTER(vp)]),
    ("mk_wcc_destroy", _S, [vp]),
    ("mk_graphset_create", _S, [C.c_uint32, u32p, C.POINTER(u32p), C.c_double, C.c_uint32,
                                C.c_int32, C.c_uint64, C.POINTER(vp)]),
    ("mk_graphset_destroy", _S, [vp]),
    ("mk_graphset_union", _S, [vp, C.POINTER(vp)]),
    ("mk_graphset_num_graphs", _S, [vp, u32p]),
    ("mk_graphset_offsets", _S, [vp, u32p]),
    ("mk_graphset_select_bits", _S, [vp, vp, vp, vp]),
    ("mk_graphset_offsets_device", _S, [vp, C.POINTER(vp)]),
    ("mk_gen_rmat_set", _S, [vp, C.c_uint32, vp, C.c_double, C.c_double, C.c_double, C.c_uint64,
                             C.c_uint32, C.c_uint32, vp, vp, vp, vp]),
    ("mk_gen_set_batches", _S, [vp, C.c_uint32, vp, vp, vp, vp, C.c_uint64, C.c_uint32, C.c_uint32,
                                vp, vp, vp, vp, vp, vp]),
    ("mk_set_runner_create", _S, [vp, vp, vp, C.POINTER(vp)]),
    ("mk_set_runner_step", _S, [vp, vp, vp, C.c_uint32, vp, vp, vp, C.c_uint32, vp]),
    ("mk_set_runner_results", _S, [vp, C.POINTER(vp), C.POINTER(vp)]),
    ("mk_set_runner_launches", _S, [vp, u32p]),
    ("mk_set_runner_set_single", _S, [vp, C.c_uint32]),
    ("mk_set_runner_handles", _S, [vp, C.POINTER(vp), C.POINTER(vp)]),
    ("mk_set_runner_destroy", _S, [vp]),
    ("mk_read_edge_list", _S, [C.c_char_p, u32p, u64p, vp, vp]),
    ("mk_read_batch_file", _S, [C.c_char_p, u64p, vp, vp]),
    ("mk_write_edge_list", _S, [C.c_char_p, C.c_uint32, C.c_uint64, vp, vp]),
    ("mk_write_batch_file", _S, [C.c_char_p, C.c_uint64, vp, vp]),
    ("mk_gen_rmat", _S, [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64,
                         C.c_uint32, C.c_uint32, vp, vp, vp]),
    ("mk_gen_grid", _S, [C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, vp, vp, vp,
                         u64p]),
    ("mk_edgeset_create", _S, [C.c_uint32, vp, vp, C.c_uint64, C.POINTER(vp)]),
    ("mk_edgeset_destroy", _S, [vp]),
    ("mk_edgeset_size", C.c_uint64, [vp]),
    ("mk_edgeset_sample_absent", _S, [vp, C.c_uint64, C.c_uint64, vp, vp]),
    ("mk_edgeset_sample_present", _S, [vp, C.c_uint64, C.c_uint64, vp, vp]),
]

_lib = None


class MeerkatError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib() -> C.CDLL:
    """Loads the CUDA library; fails loudly when it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m meerkat_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != MK_OK:
        msg = lib().mk_last_error_string().decode(errors="replace")
        raise MeerkatError(status, where, msg)
