"""ctypes bindings of libblest_b200.so (the C ABI declared in include/blest.h).

The shared library is built in-tree (python blest_b200/build.py). There is
no Python or CPU fallback for the device entry points: if the library is
missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libblest_b200.so"

if not LIB_PATH.exists():
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python blest_b200/build.py` "
        "(the BFS/CC/MBFS path has no CPU fallback)")

lib = C.CDLL(str(LIB_PATH))

u8, u32, u64, i32, f64 = C.c_uint8, C.c_uint32, C.c_uint64, C.c_int, C.c_double
P = C.POINTER
vp = C.c_void_p

OK = 0
ERR_INVALID_ARG = 1
ERR_CUDA = 2
ERR_OOM = 3
ERR_LEVEL_CAP = 4
ERR_BARRIER_TIMEOUT = 5
ERR_NO_DEVICE = 6
ERR_UNSUPPORTED = 7
ERR_IO = 8
ERR_ADMISSION = 9
ERR_DEVICE_INDEX = 10
ERR_BUSY = 11
UNREACHED = 0xFFFFFFFF
NOALLOC_MAX_VERTICES = 1 << 20
MEM_HOST = 0
MEM_DEVICE = 1

ORDER_AUTO, ORDER_NATURAL, ORDER_JACCARD, ORDER_RCM, ORDER_RANDOM, ORDER_DEGREE, ORDER_GORDER = range(7)
DIR_AUTO, DIR_PUSH, DIR_PULL = 0, 1, 2
QUERY_BFS, QUERY_CC = 0, 1
TEST_CUDA_CORE, TEST_B1_MMA = 0, 1


class BlestError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[blest error {code}] {msg}")
        self.code = code


class CscView(C.Structure):
    _fields_ = [("n", u32), ("nnz", u32), ("is_social", i32), ("col_ptrs", P(u32)), ("rows", P(u32))]


class OrderParams(C.Structure):
    _fields_ = [("mode", i32), ("jaccard_enabled", i32), ("window", u32), ("seed", u64),
                ("rcm_rand_seed", u32), ("threads", i32)]


class BvssView(C.Structure):
    _fields_ = [("n", u32), ("slice_size", u32), ("no_masks", u32), ("no_real_slice_sets", u32),
                ("no_virtual_slice_sets", u32), ("no_slices", u64), ("no_padded_slices", u64),
                ("update_divergence", f64), ("full_padding", i32), ("slice_set_ptrs", P(u64)),
                ("virtual_to_real", P(u32)), ("real_ptrs", P(u32)), ("row_ids", P(u32)), ("masks", P(u32))]


class CsrView(C.Structure):
    _fields_ = [("n", u32), ("nnz", u32), ("row_ptrs", P(u32)), ("col_ids", P(u32))]


class GraphInfo(C.Structure):
    _fields_ = [("n", u32), ("no_real_slice_sets", u32), ("no_virtual_slice_sets", u32), ("no_slices", u64),
                ("nnz", u32), ("undirected_edges", u64), ("device_bytes_graph", u64),
                ("device_bytes_workspace", u64), ("device", i32), ("device_tiles", u64)]


class BfsParams(C.Structure):
    _fields_ = [("direction", i32), ("slice_test", i32), ("alpha", f64), ("beta", f64),
                ("blocks_per_sm", i32), ("threads_per_block", i32), ("trace", i32)]


class LevelTrace(C.Structure):
    _fields_ = [("start_ns", u64), ("level", u32), ("direction", u32), ("frontier", u64), ("work_units", u64),
                ("longest_scan", u64), ("sweep_ns", u64)]


class BfsStats(C.Structure):
    _fields_ = [("time", f64), ("source_vertex", u32), ("total_levels", u32), ("no_visited", u32),
                ("push_levels", u32), ("pull_levels", u32), ("reached_degree_sum", u64)]


class CcStats(C.Structure):
    _fields_ = [("time", f64), ("no_components", u32), ("iterations", u32)]


class DeviceGraphView(C.Structure):
    _fields_ = [("n", u32), ("no_real_slice_sets", u32), ("no_slices", u64), ("nnz", u32),
                ("slice_set_ptrs", vp), ("real_ptrs", vp), ("row_ids", vp), ("masks", vp),
                ("csr_ptrs", vp), ("csr_ids", vp)]


class MbfsParams(C.Structure):
    _fields_ = [("group_width", u32), ("blocks_per_sm", i32), ("threads_per_block", i32), ("pull_fraction", f64),
                ("trace", i32)]


class MbfsStats(C.Structure):
    _fields_ = [("time", f64), ("groups", u32), ("max_levels", u32), ("reached_degree_sum", u64)]


class ServerParams(C.Structure):
    _fields_ = [("memory_budget", u64), ("lanes", u32), ("max_batch", u32), ("queue_capacity", u32),
                ("dry_run", i32), ("completion_queue", i32), ("batch_policy", i32)]


class QueryResult(C.Structure):
    _fields_ = [("status", i32), ("kind", i32), ("graph_id", u32), ("source", u32), ("batch_size", u32),
                ("submit_s", f64), ("start_s", f64), ("done_s", f64)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", u64), ("completed", u64), ("rejected", u64), ("jobs", u64),
                ("batched_requests", u64), ("p50_latency_s", f64), ("p99_latency_s", f64),
                ("mean_latency_s", f64), ("busy_s", f64), ("peak_reserved_bytes", u64), ("memory_budget", u64),
                ("jobs_bfs", u64), ("jobs_mbfs", u64), ("jobs_cc", u64), ("requests_mbfs", u64),
                ("requests_cc", u64), ("busy_bfs_s", f64), ("busy_mbfs_s", f64), ("busy_cc_s", f64),
                ("unbatched_requests", u64)]


class MbfsItem(C.Structure):
    _fields_ = [("graph", vp), ("sources", P(u32)), ("k", u32), ("levels_out", vp)]


class MbfsPlanInfo(C.Structure):
    _fields_ = [("items", u32), ("n", u32), ("nnz", u64), ("no_slices", u64), ("groups", u32),
                ("group_width", u32), ("grid_blocks", i32), ("captured", i32), ("device_bytes", u64)]


def _sig(name, args, res=i32):
    f = getattr(lib, name, None)
    if f is None:
        return None
    f.argtypes = args
    f.restype = res
    return f


_SIGS = {
    "blest_init": [i32],
    "blest_last_error": ([], C.c_char_p),
    "blest_version": ([], C.c_char_p),
    "blest_csc_read_mtx": [C.c_char_p, i32, i32, P(vp)],
    "blest_csc_read_mtx_auto": [C.c_char_p, P(vp)],
    "blest_csc_load_bin": [C.c_char_p, P(vp)],
    "blest_csc_save_bin": [vp, C.c_char_p],
    "blest_csc_from_arrays": [u32, P(u32), P(u32), P(vp)],
    "blest_csc_generate_rmat": [u32, u32, f64, f64, f64, u64, u64, P(vp)],
    "blest_csc_generate_grid": [u32, u32, f64, f64, u64, u64, P(vp)],
    "blest_csc_generate_er": [u32, u64, u64, u64, P(vp)],
    "blest_csc_view_get": [vp, P(CscView)],
    "blest_csc_destroy": [vp],
    "blest_csc_transpose": [vp, P(vp)],
    "blest_csc_check_symmetry": [vp, P(i32)],
    "blest_csc_symmetrize": [vp, P(vp)],
    "blest_csc_sample_sources": [vp, u32, u64, P(u32), P(u32)],
    "blest_csc_reorder": [vp, P(OrderParams), P(u32)],
    "blest_csc_apply_permutation": [vp, P(u32)],
    "blest_ordering_save_bin": [C.c_char_p, P(u32), u32],
    "blest_ordering_load_bin": [C.c_char_p, u32, P(u32)],
    "blest_bvss_build": [vp, i32, P(vp)],
    "blest_bvss_from_view": [P(BvssView), P(vp)],
    "blest_bvss_view_get": [vp, P(BvssView)],
    "blest_bvss_save_bin": [vp, C.c_char_p],
    "blest_bvss_load_bin": [C.c_char_p, P(vp)],
    "blest_bvss_destroy": [vp],
    "blest_bvss_build_device": [vp, i32, P(vp)],
    "blest_bvss_edge_check": [vp, P(u64)],
    "blest_graph_create": [P(BvssView), P(CsrView), P(vp)],
    "blest_graph_create_from_csc": [vp, vp, i32, P(vp)],
    "blest_graph_destroy": [vp],
    "blest_graph_info_get": [vp, P(GraphInfo)],
    "blest_graph_set_stream": [vp, vp],
    "blest_workspace_create": [vp, P(vp)],
    "blest_workspace_destroy": [vp],
    "blest_bfs": [vp, u32, vp, vp, i32, P(BfsParams), P(BfsStats)],
    "blest_bfs_ws": [vp, u32, vp, vp, i32, P(BfsParams), vp, i32, P(BfsStats)],
    "blest_workspace_sync": [vp, P(BfsStats)],
    "blest_workspace_sync_one": [vp, P(i32), P(BfsStats)],
    "blest_workspace_trace": [vp, P(LevelTrace), u32, P(u32)],
    "blest_graph_default_workspace": [vp, P(vp)],
    "blest_bfs_noalloc": [P(DeviceGraphView), u32, vp, vp, vp, P(BfsStats)],
    "blest_selftest_barrier": [u32, u32, u64, u32, P(f64)],
    "blest_cc": [vp, vp, i32, P(CcStats)],
    "blest_cc_ws": [vp, vp, i32, vp, P(CcStats)],
    "blest_cc_relabel_dense": [P(u32), u32, P(u32), P(u32)],
    "blest_mbfs": [vp, P(u32), u32, vp, i32, P(MbfsParams), P(MbfsStats)],
    "blest_mbfs_batch": [P(MbfsItem), u32, i32, P(MbfsParams), vp, P(MbfsStats)],
    "blest_mbfs_ws": [vp, P(u32), u32, vp, i32, P(MbfsParams), vp, P(MbfsStats)],
    "blest_mbfs_rows_ws": [vp, P(u32), u32, P(vp), P(MbfsParams), vp, P(MbfsStats)],
    "blest_mbfs_plan_create": [P(MbfsItem), u32, P(MbfsParams), vp, P(vp)],
    "blest_mbfs_plan_set_sources": [vp, u32, P(u32)],
    "blest_mbfs_plan_run": [vp, P(MbfsStats)],
    "blest_mbfs_plan_launch": [vp],
    "blest_mbfs_plan_sync": [vp, P(MbfsStats)],
    "blest_mbfs_plan_info_get": [vp, P(MbfsPlanInfo)],
    "blest_mbfs_plan_destroy": [vp],
    "blest_workspace_set_grid": [vp, u32],
    "blest_server_create": [P(ServerParams), P(vp)],
    "blest_server_add_graph": [vp, vp, P(u32)],
    "blest_server_add_virtual_graph": [vp, u32, u64, P(u32)],
    "blest_server_submit": [vp, u32, i32, u32, vp, P(u64)],
    "blest_server_submit_ex": [vp, u32, i32, u32, vp, i32, P(u64)],
    "blest_server_poll": [vp, u64, P(i32), P(QueryResult)],
    "blest_server_wait": [vp, u64, f64, P(QueryResult)],
    "blest_server_drain": [vp, f64],
    "blest_server_next_done": [vp, f64, P(u64), P(QueryResult)],
    "blest_server_release": [vp, u64],
    "blest_server_stats_get": [vp, P(ServerStats)],
    "blest_server_destroy": [vp],
}

fn = {}
for _name, _spec in _SIGS.items():
    if isinstance(_spec, tuple):
        fn[_name] = _sig(_name, _spec[0], _spec[1])
    else:
        fn[_name] = _sig(_name, _spec)


def declared_symbols() -> list[str]:
    """Every function name declared in include/*.h (parsed from the headers)."""
    import re
    names = []
    for h in sorted((_PKG.parent / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[\w]+\s*\**\s*(blest_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def check(rc: int) -> None:
    if rc != OK:
        msg = lib.blest_last_error().decode(errors="replace")
        raise BlestError(rc, msg)


def call(name: str, *args) -> None:
    f = fn.get(name)
    if f is None:
        raise BlestError(ERR_UNSUPPORTED, f"{name} is not exported by {LIB_PATH.name}")
    check(f(*args))
