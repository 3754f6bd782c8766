"""Host-side objects over the C ABI: CSC / BVSS (CPU preprocessing) and the
device-resident Graph with its BFS / CC / MBFS entry points."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L

_ORDER_MODES = {"auto": L.ORDER_AUTO, "natural": L.ORDER_NATURAL, "jaccard": L.ORDER_JACCARD,
                "rcm": L.ORDER_RCM, "random": L.ORDER_RANDOM, "degree": L.ORDER_DEGREE,
                "gorder": L.ORDER_GORDER}


def _destroy(name: str, h) -> None:
    """Free a handle; at interpreter shutdown the bindings may already be
    gone, and the process exit releases the memory anyway."""
    try:
        L.fn[name](h)
    except (TypeError, AttributeError, KeyError):
        pass


def _u32p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(L.P(L.u32))


def _u64p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(L.P(L.u64))


def _view(ptr, count: int, dtype) -> np.ndarray:
    if count == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(count,)).view(dtype)


class Csc:
    """Column-compressed graph (column = source vertex; rows = out-neighbours),
    DataStructures/CSC.cuh. Array properties are zero-copy views valid while
    this object lives and is not reordered."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("blest_csc_destroy", h)
            self._h = None

    @staticmethod
    def _make(name: str, *args) -> "Csc":
        h = C.c_void_p()
        L.call(name, *args, C.byref(h))
        return Csc(h)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1, permute_seed: int = 1) -> "Csc":
        return cls._make("blest_csc_generate_rmat", scale, edge_factor, a, b, c, seed, permute_seed)

    @classmethod
    def grid(cls, width: int, height: int, p_delete: float = 0.05, shortcut_fraction: float = 0.001,
             seed: int = 1, permute_seed: int = 0) -> "Csc":
        return cls._make("blest_csc_generate_grid", width, height, p_delete, shortcut_fraction, seed, permute_seed)

    @classmethod
    def er(cls, n: int, m: int, seed: int = 1, permute_seed: int = 0) -> "Csc":
        return cls._make("blest_csc_generate_er", n, m, seed, permute_seed)

    @classmethod
    def from_arrays(cls, n: int, col_ptrs, rows) -> "Csc":
        cp = np.ascontiguousarray(col_ptrs, dtype=np.uint32)
        rw = np.ascontiguousarray(rows, dtype=np.uint32)
        if rw.size == 0:
            rw = np.zeros(1, dtype=np.uint32)
        return cls._make("blest_csc_from_arrays", n, _u32p(cp), _u32p(rw))

    @classmethod
    def from_edges(cls, n: int, src, dst) -> "Csc":
        """Directed edges src[i] -> dst[i] (no dedup; self loops kept)."""
        src = np.asarray(src, dtype=np.int64)
        dst = np.asarray(dst, dtype=np.int64)
        order = np.lexsort((dst, src))
        src, dst = src[order], dst[order]
        col_ptrs = np.zeros(n + 1, dtype=np.uint32)
        np.add.at(col_ptrs, src + 1, 1)
        col_ptrs = np.cumsum(col_ptrs, dtype=np.uint64).astype(np.uint32)
        return cls.from_arrays(n, col_ptrs, dst.astype(np.uint32))

    @classmethod
    def read_mtx(cls, path: str, undirected: bool | None = None, binary: bool | None = None) -> "Csc":
        if undirected is None or binary is None:
            return cls._make("blest_csc_read_mtx_auto", str(path).encode())
        return cls._make("blest_csc_read_mtx", str(path).encode(), int(undirected), int(binary))

    @classmethod
    def load_bin(cls, path: str) -> "Csc":
        return cls._make("blest_csc_load_bin", str(path).encode())

    def save_bin(self, path: str) -> None:
        L.call("blest_csc_save_bin", self._h, str(path).encode())

    def _v(self) -> L.CscView:
        v = L.CscView()
        L.call("blest_csc_view_get", self._h, C.byref(v))
        return v

    @property
    def n(self) -> int:
        return self._v().n

    @property
    def nnz(self) -> int:
        return self._v().nnz

    @property
    def is_social(self) -> bool:
        return bool(self._v().is_social)

    @property
    def col_ptrs(self) -> np.ndarray:
        v = self._v()
        return _view(v.col_ptrs, v.n + 1, np.uint32)

    @property
    def rows(self) -> np.ndarray:
        v = self._v()
        return _view(v.rows, v.nnz, np.uint32)

    def degrees(self) -> np.ndarray:
        return np.diff(self.col_ptrs.astype(np.int64)).astype(np.uint32)

    def transpose(self) -> "Csc":
        return self._make("blest_csc_transpose", self._h)

    def symmetrize(self) -> "Csc":
        return self._make("blest_csc_symmetrize", self._h)

    def is_symmetric(self) -> bool:
        s = C.c_int()
        L.call("blest_csc_check_symmetry", self._h, C.byref(s))
        return bool(s.value)

    def sample_sources(self, k: int, seed: int) -> np.ndarray:
        out = np.zeros(max(k, 1), dtype=np.uint32)
        cnt = L.u32()
        L.call("blest_csc_sample_sources", self._h, k, seed, _u32p(out), C.byref(cnt))
        return out[: cnt.value].copy()

    def reorder(self, mode: str = "auto", jaccard: bool = True, window: int = 65536, seed: int = 0,
                rcm_rand_seed: int = 1, threads: int = 0) -> np.ndarray:
        """Compute + apply an ordering (CSC::reorder, CSC.cuh:358-386);
        returns inversePermutation (inv[old] = new)."""
        p = L.OrderParams(_ORDER_MODES[mode], int(jaccard), window, seed, rcm_rand_seed, threads)
        inv = np.zeros(self.n, dtype=np.uint32)
        L.call("blest_csc_reorder", self._h, C.byref(p), _u32p(inv))
        return inv

    def apply_permutation(self, inv) -> None:
        inv = np.ascontiguousarray(inv, dtype=np.uint32)
        L.call("blest_csc_apply_permutation", self._h, _u32p(inv))


def save_ordering(path: str, inv: np.ndarray) -> None:
    inv = np.ascontiguousarray(inv, dtype=np.uint32)
    L.call("blest_ordering_save_bin", str(path).encode(), _u32p(inv), inv.size)


def load_ordering(path: str, n: int) -> np.ndarray:
    inv = np.zeros(n, dtype=np.uint32)
    L.call("blest_ordering_load_bin", str(path).encode(), n, _u32p(inv))
    return inv


class Bvss:
    """Bit-Vector Slice Sets (DataStructures/BVSS.cuh). Array properties are
    zero-copy views valid while this object lives."""

    def __init__(self, handle: C.c_void_p, keep=None):
        self._h = handle
        self._keep = keep

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("blest_bvss_destroy", h)
            self._h = None

    @classmethod
    def build(cls, csc: Csc, full_padding: bool | None = None) -> "Bvss":
        h = C.c_void_p()
        fp = -1 if full_padding is None else int(full_padding)
        L.call("blest_bvss_build", csc._h, fp, C.byref(h))
        return cls(h)

    @classmethod
    def build_device(cls, csc: Csc, full_padding: bool | None = None) -> "Bvss":
        """The same BVSS built by GPU kernels (blest_bvss_build_device)."""
        if not _initialised:
            init(0)
        h = C.c_void_p()
        fp = -1 if full_padding is None else int(full_padding)
        L.call("blest_bvss_build_device", csc._h, fp, C.byref(h))
        return cls(h)

    @classmethod
    def load_bin(cls, path: str) -> "Bvss":
        h = C.c_void_p()
        L.call("blest_bvss_load_bin", str(path).encode(), C.byref(h))
        return cls(h)

    @classmethod
    def from_arrays(cls, n, slice_set_ptrs, virtual_to_real, real_ptrs, row_ids, masks,
                    full_padding=False, update_divergence=0.0) -> "Bvss":
        ssp = np.ascontiguousarray(slice_set_ptrs, dtype=np.uint64)
        v2r = np.ascontiguousarray(virtual_to_real, dtype=np.uint32)
        rp = np.ascontiguousarray(real_ptrs, dtype=np.uint32)
        ri = np.ascontiguousarray(row_ids, dtype=np.uint32)
        mk = np.ascontiguousarray(masks, dtype=np.uint32)
        keep = [np.concatenate([a, np.zeros(1, a.dtype)]) if a.size == 0 else a for a in (v2r, ri, mk)]
        v = L.BvssView(n, 8, 4, rp.size - 1, v2r.size, ri.size, 0, update_divergence, int(full_padding),
                       _u64p(ssp), _u32p(keep[0]), _u32p(rp), _u32p(keep[1]), _u32p(keep[2]))
        h = C.c_void_p()
        L.call("blest_bvss_from_view", C.byref(v), C.byref(h))
        return cls(h)

    def save_bin(self, path: str) -> None:
        L.call("blest_bvss_save_bin", self._h, str(path).encode())

    def view(self) -> L.BvssView:
        v = L.BvssView()
        L.call("blest_bvss_view_get", self._h, C.byref(v))
        return v

    def arrays(self) -> dict:
        v = self.view()
        return {
            "slice_set_ptrs": _view(v.slice_set_ptrs, v.no_virtual_slice_sets + 1, np.uint64),
            "virtual_to_real": _view(v.virtual_to_real, v.no_virtual_slice_sets, np.uint32),
            "real_ptrs": _view(v.real_ptrs, v.no_real_slice_sets + 1, np.uint32),
            "row_ids": _view(v.row_ids, v.no_slices, np.uint32),
            "masks": _view(v.masks, v.no_slices // 4, np.uint32),
        }

    def edge_check(self) -> int:
        e = L.u64()
        L.call("blest_bvss_edge_check", self._h, C.byref(e))
        return e.value

    @property
    def n(self) -> int:
        return self.view().n

    @property
    def update_divergence(self) -> float:
        return self.view().update_divergence

    @property
    def full_padding(self) -> bool:
        return bool(self.view().full_padding)


@dataclass
class BfsStats:
    time: float
    source_vertex: int
    total_levels: int
    no_visited: int
    push_levels: int
    pull_levels: int
    reached_degree_sum: int


@dataclass
class CcStats:
    time: float
    no_components: int
    iterations: int


@dataclass
class MbfsStats:
    time: float
    groups: int
    max_levels: int
    reached_degree_sum: int


_initialised = False


def init(device: int = 0) -> None:
    global _initialised
    L.call("blest_init", device)
    _initialised = True


def bfs_params(direction: str = "auto", slice_test: str = "cuda_core", alpha: float = 0.0, beta: float = 0.0,
               blocks_per_sm: int = 0, threads_per_block: int = 0, trace: bool = False) -> L.BfsParams:
    d = {"auto": L.DIR_AUTO, "push": L.DIR_PUSH, "pull": L.DIR_PULL}[direction]
    t = {"cuda_core": L.TEST_CUDA_CORE, "mma": L.TEST_B1_MMA}[slice_test]
    return L.BfsParams(d, t, alpha, beta, blocks_per_sm, threads_per_block, int(trace))


class Graph:
    """A graph resident in HBM (BVSS + pull CSR), blest_graph_create."""

    def __init__(self, bvss: Bvss, csr: Csc):
        if not _initialised:
            init(0)
        v = bvss.view()
        cv = csr._v()
        cs = L.CsrView(cv.n, cv.nnz, cv.col_ptrs, cv.rows)
        h = C.c_void_p()
        L.call("blest_graph_create", C.byref(v), C.byref(cs), C.byref(h))
        self._h = h
        self.n = v.n

    @classmethod
    def from_csc(cls, csc: Csc, csr: Csc | None = None, full_padding: bool | None = None) -> "Graph":
        """Resident graph whose BVSS is built on the device from `csc`
        (blest_graph_create_from_csc); `csr` = pull CSR, None for a
        symmetric CSC."""
        if not _initialised:
            init(0)
        g = cls.__new__(cls)
        h = C.c_void_p()
        fp = -1 if full_padding is None else int(full_padding)
        L.call("blest_graph_create_from_csc", csc._h, csr._h if csr is not None else None, fp, C.byref(h))
        g._h = h
        g.n = csc.n
        return g

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            _destroy("blest_graph_destroy", h)
            self._h = None

    __del__ = close

    def trace(self) -> list[dict]:
        """Per-level records of the last BFS run with bfs_params(trace=True)."""
        ws = C.c_void_p()
        L.call("blest_graph_default_workspace", self._h, C.byref(ws))
        recs = (L.LevelTrace * 4096)()
        cnt = L.u32()
        L.call("blest_workspace_trace", ws, recs, 4096, C.byref(cnt))
        out = []
        for i in range(cnt.value):
            r = recs[i]
            out.append({"level": r.level, "dir": {1: "push", 2: "pull", 3: "both"}.get(r.direction, "end"),
                        "start_ns": r.start_ns, "frontier": r.frontier, "work_units": r.work_units,
                        "longest_scan": r.longest_scan})
        return out

    def info(self) -> L.GraphInfo:
        i = L.GraphInfo()
        L.call("blest_graph_info_get", self._h, C.byref(i))
        return i

    def bfs(self, source: int, parents: bool = False, params: L.BfsParams | None = None):
        """BFS from `source`: returns (levels, parents-or-None, BfsStats)."""
        lv = np.empty(self.n, dtype=np.uint32)
        pa = np.empty(self.n, dtype=np.uint32) if parents else None
        st = L.BfsStats()
        L.call("blest_bfs", self._h, source, lv.ctypes.data, pa.ctypes.data if parents else None, L.MEM_HOST,
               C.byref(params) if params is not None else None, C.byref(st))
        return lv, pa, BfsStats(st.time, st.source_vertex, st.total_levels, st.no_visited, st.push_levels,
                                st.pull_levels, st.reached_degree_sum)

    def bfs_device(self, source: int, levels_ptr: int, parents_ptr: int | None = None,
                   params: L.BfsParams | None = None) -> BfsStats:
        """BFS writing levels to a device buffer (e.g. a torch tensor's data_ptr())."""
        st = L.BfsStats()
        L.call("blest_bfs", self._h, source, levels_ptr, parents_ptr, L.MEM_DEVICE,
               C.byref(params) if params is not None else None, C.byref(st))
        return BfsStats(st.time, st.source_vertex, st.total_levels, st.no_visited, st.push_levels,
                        st.pull_levels, st.reached_degree_sum)

    def cc(self):
        """Connected components: returns (labels, CcStats); labels[v] = min id reaching v."""
        lab = np.empty(self.n, dtype=np.uint32)
        st = L.CcStats()
        L.call("blest_cc", self._h, lab.ctypes.data, L.MEM_HOST, C.byref(st))
        return lab, CcStats(st.time, st.no_components, st.iterations)

    def mbfs(self, sources, group_width: int = 128, blocks_per_sm: int = 0, threads_per_block: int = 0,
             pull_fraction: float = 0.0, trace: bool = False):
        """Multi-source BFS: returns (levels[k, n], MbfsStats)."""
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        out = np.empty((src.size, self.n), dtype=np.uint32)
        p = L.MbfsParams(group_width, blocks_per_sm, threads_per_block, pull_fraction, int(trace))
        st = L.MbfsStats()
        L.call("blest_mbfs", self._h, _u32p(src), src.size, out.ctypes.data, L.MEM_HOST, C.byref(p), C.byref(st))
        return out, MbfsStats(st.time, st.groups, st.max_levels, st.reached_degree_sum)


def relabel_dense(labels: np.ndarray):
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    out = np.empty_like(lab)
    k = L.u32()
    L.call("blest_cc_relabel_dense", _u32p(lab), lab.size, _u32p(out), C.byref(k))
    return out, k.value


class Workspace:
    """Per-query scratch on a Graph (blest_workspace_create), for
    concurrent or asynchronous queries on explicit streams."""

    def __init__(self, graph: Graph):
        h = C.c_void_p()
        L.call("blest_workspace_create", graph._h, C.byref(h))
        self._h = h
        self.graph = graph

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            _destroy("blest_workspace_destroy", h)
            self._h = None

    __del__ = close

    def bfs_async(self, source: int, levels_ptr: int, stream: int, parents_ptr: int | None = None,
                  params: L.BfsParams | None = None, out_mem: int = L.MEM_DEVICE) -> None:
        """Enqueue a BFS on `stream` (a cudaStream_t as int); returns at once.
        With out_mem=MEM_HOST (a pinned buffer that must stay untouched until
        the call is settled) the copy overlaps the next call's kernel."""
        L.call("blest_bfs_ws", self._h, source, levels_ptr, parents_ptr, out_mem,
               C.byref(params) if params is not None else None, stream, 1, None)

    def sync(self) -> BfsStats:
        """Settle every pending asynchronous call (first failure raised);
        returns the last call's stats."""
        st = L.BfsStats()
        L.call("blest_workspace_sync", self._h, C.byref(st))
        return BfsStats(st.time, st.source_vertex, st.total_levels, st.no_visited, st.push_levels,
                        st.pull_levels, st.reached_degree_sum)

    def sync_one(self) -> BfsStats | None:
        """Settle the oldest pending call only (None when nothing is pending)."""
        st = L.BfsStats()
        done = L.i32()
        L.call("blest_workspace_sync_one", self._h, C.byref(done), C.byref(st))
        if not done.value:
            return None
        return BfsStats(st.time, st.source_vertex, st.total_levels, st.no_visited, st.push_levels,
                        st.pull_levels, st.reached_degree_sum)

    def bfs(self, source: int, levels_out: np.ndarray, stream: int = 0, params: L.BfsParams | None = None):
        """Blocking BFS into a host array (pinned or pageable); returns BfsStats."""
        st = L.BfsStats()
        L.call("blest_bfs_ws", self._h, source, levels_out.ctypes.data, None, L.MEM_HOST,
               C.byref(params) if params is not None else None, stream, 0, C.byref(st))
        return BfsStats(st.time, st.source_vertex, st.total_levels, st.no_visited, st.push_levels,
                        st.pull_levels, st.reached_degree_sum)

    def cc(self, labels_ptr: int, stream: int = 0, out_mem: int = L.MEM_DEVICE) -> CcStats:
        st = L.CcStats()
        L.call("blest_cc_ws", self._h, labels_ptr, out_mem, stream, C.byref(st))
        return CcStats(st.time, st.no_components, st.iterations)

    def mbfs_rows(self, sources, rows, group_width: int = 128, stream: int = 0) -> MbfsStats:
        """Blocking multi-source BFS with one device buffer per source:
        rows[i] (a device pointer as int) receives the n levels of
        sources[i] (blest_mbfs_rows_ws)."""
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        assert len(rows) == src.size
        ptrs = (C.c_void_p * max(1, src.size))(*rows)
        p = L.MbfsParams(group_width, 0, 0, 0.0, 0)
        st = L.MbfsStats()
        L.call("blest_mbfs_rows_ws", self._h, _u32p(src), src.size, ptrs, C.byref(p), stream, C.byref(st))
        return MbfsStats(st.time, st.groups, st.max_levels, st.reached_degree_sum)


class MbfsPlan:
    """Multi-graph multi-source BFS in one persistent launch, replayed from a
    captured CUDA graph (blest_mbfs_plan_*). `items` is a list of
    (Graph, sources, levels_ptr): levels_ptr is device memory holding
    k * n uint32 levels (source-major) for that graph."""

    def __init__(self, items, group_width: int = 32, blocks_per_sm: int = 0, threads_per_block: int = 0,
                 pull_fraction: float = 0.0, stream: int | None = None):
        self._srcs = [np.ascontiguousarray(s, dtype=np.uint32) for _, s, _ in items]
        arr = (L.MbfsItem * len(items))()
        for i, ((g, _, ptr), src) in enumerate(zip(items, self._srcs)):
            arr[i] = L.MbfsItem(g._h, _u32p(src), src.size, ptr)
        self.graphs = [g for g, _, _ in items]
        p = L.MbfsParams(group_width, blocks_per_sm, threads_per_block, pull_fraction)
        h = C.c_void_p()
        L.call("blest_mbfs_plan_create", arr, len(items), C.byref(p), stream, C.byref(h))
        self._h = h

    def set_sources(self, item: int, sources) -> None:
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        L.call("blest_mbfs_plan_set_sources", self._h, item, _u32p(src))

    def run(self) -> MbfsStats:
        st = L.MbfsStats()
        L.call("blest_mbfs_plan_run", self._h, C.byref(st))
        return MbfsStats(st.time, st.groups, st.max_levels, st.reached_degree_sum)

    def launch(self) -> None:
        L.call("blest_mbfs_plan_launch", self._h)

    def sync(self) -> MbfsStats:
        st = L.MbfsStats()
        L.call("blest_mbfs_plan_sync", self._h, C.byref(st))
        return MbfsStats(st.time, st.groups, st.max_levels, st.reached_degree_sum)

    def info(self) -> L.MbfsPlanInfo:
        i = L.MbfsPlanInfo()
        L.call("blest_mbfs_plan_info_get", self._h, C.byref(i))
        return i

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            _destroy("blest_mbfs_plan_destroy", h)
            self._h = None

    __del__ = close


def mbfs_batch(items, out_mem: int = L.MEM_HOST, group_width: int = 32, blocks_per_sm: int = 0,
               pull_fraction: float = 0.0) -> MbfsStats:
    """blest_mbfs_batch over [(Graph, sources, levels)] where levels is a
    (k, n) uint32 numpy array (out_mem host) or a device pointer."""
    srcs = [np.ascontiguousarray(s, dtype=np.uint32) for _, s, _ in items]
    arr = (L.MbfsItem * len(items))()
    for i, ((g, _, out), src) in enumerate(zip(items, srcs)):
        ptr = out.ctypes.data if isinstance(out, np.ndarray) else out
        arr[i] = L.MbfsItem(g._h, _u32p(src), src.size, ptr)
    p = L.MbfsParams(group_width, blocks_per_sm, 0, pull_fraction)
    st = L.MbfsStats()
    L.call("blest_mbfs_batch", arr, len(items), out_mem, C.byref(p), None, C.byref(st))
    return MbfsStats(st.time, st.groups, st.max_levels, st.reached_degree_sum)
