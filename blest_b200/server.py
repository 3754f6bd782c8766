"""Query server with continuous batching (blest_server_* in include/blest.h).

    srv = Server(lanes=4)
    gid = srv.add_graph(graph)                 # a resident blest_b200.Graph
    t = srv.submit_bfs(gid, source)            # returns a Ticket
    levels = t.result()                        # numpy uint32[n]
    srv.stats()                                # p50 / p99 latency, jobs, batching

With completion_queue=True, srv.next_done() returns finished tickets in
completion order, so a client can reuse each result buffer as soon as its
request is done.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class QueryInfo:
    status: int
    kind: str
    graph_id: int
    source: int
    batch_size: int
    submit_s: float
    start_s: float
    done_s: float

    @property
    def latency_s(self) -> float:
        return self.done_s - self.submit_s


class Ticket:
    def __init__(self, server: "Server", ticket: int, out: np.ndarray):
        self.server = server
        self.id = ticket
        self.out = out

    def done(self) -> bool:
        d = C.c_int()
        L.call("blest_server_poll", self.server._h, self.id, C.byref(d), None)
        return bool(d.value)

    def info(self, timeout_s: float = 600.0) -> QueryInfo:
        r = L.QueryResult()
        rc = L.fn["blest_server_wait"](self.server._h, self.id, timeout_s, C.byref(r))
        if rc not in (L.OK,) and r.status == L.OK:
            L.check(rc)
        return QueryInfo(r.status, {0: "bfs", 1: "cc"}.get(r.kind, "?"), r.graph_id, r.source, r.batch_size,
                         r.submit_s, r.start_s, r.done_s)

    def result(self, timeout_s: float = 600.0) -> np.ndarray:
        r = L.QueryResult()
        L.call("blest_server_wait", self.server._h, self.id, timeout_s, C.byref(r))
        return self.out


class Server:
    def __init__(self, lanes: int = 4, max_batch: int = 128, memory_budget: int = 0, queue_capacity: int = 0,
                 dry_run: bool = False, completion_queue: bool = False, always_batch: bool = False):
        """always_batch: coalesce every group of pending BFS requests on a
        graph (BLEST_BATCH_ALWAYS) instead of the adaptive policy."""
        p = L.ServerParams(memory_budget, lanes, max_batch, queue_capacity, int(dry_run), int(completion_queue),
                           int(always_batch))
        h = C.c_void_p()
        L.call("blest_server_create", C.byref(p), C.byref(h))
        self._h = h
        self._graphs = {}
        self.dry_run = dry_run

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            L.fn["blest_server_destroy"](h)
            self._h = None

    __del__ = close

    def add_graph(self, graph) -> int:
        gid = L.u32()
        L.call("blest_server_add_graph", self._h, graph._h, C.byref(gid))
        self._graphs[gid.value] = graph  # keep it alive
        return gid.value

    def add_virtual_graph(self, n: int, nnz: int = 0) -> int:
        gid = L.u32()
        L.call("blest_server_add_virtual_graph", self._h, n, nnz, C.byref(gid))
        self._graphs[gid.value] = n
        return gid.value

    def _n(self, gid: int) -> int:
        g = self._graphs.get(gid, 1)  # unknown ids are refused by the library
        return g if isinstance(g, int) else g.n

    def _submit(self, gid: int, kind: int, source: int, out=None) -> Ticket:
        if out is None:
            out = np.empty(self._n(gid), dtype=np.uint32)
        t = L.u64()
        if isinstance(out, np.ndarray):
            assert out.dtype == np.uint32 and out.size >= self._n(gid) and out.flags.c_contiguous
            L.call("blest_server_submit_ex", self._h, gid, kind, source, out.ctypes.data, L.MEM_HOST, C.byref(t))
        else:
            # a device buffer (a CUDA tensor of >= n 4-byte elements): the
            # result stays on the GPU
            assert out.is_cuda and out.is_contiguous() and out.element_size() == 4 and out.numel() >= self._n(gid)
            L.call("blest_server_submit_ex", self._h, gid, kind, source, out.data_ptr(), L.MEM_DEVICE, C.byref(t))
        return Ticket(self, t.value, out)

    def submit_bfs(self, gid: int, source: int, out=None) -> Ticket:
        """`out`: optional result buffer, a uint32[n] numpy array (e.g. pinned
        memory) or a CUDA tensor of n int32/uint32 (the result stays on the
        device)."""
        return self._submit(gid, L.QUERY_BFS, source, out)

    def submit_cc(self, gid: int, out: np.ndarray | None = None) -> Ticket:
        return self._submit(gid, L.QUERY_CC, 0, out)

    def next_done(self, timeout_s: float = 600.0) -> tuple[int, QueryInfo] | None:
        """(ticket id, QueryInfo) of the next request to finish or be refused
        (servers made with completion_queue=True); None on timeout."""
        t = L.u64()
        r = L.QueryResult()
        rc = L.fn["blest_server_next_done"](self._h, timeout_s, C.byref(t), C.byref(r))
        if rc == L.ERR_BUSY:
            return None
        L.check(rc)
        return t.value, QueryInfo(r.status, {0: "bfs", 1: "cc"}.get(r.kind, "?"), r.graph_id, r.source,
                                  r.batch_size, r.submit_s, r.start_s, r.done_s)

    def release(self, ticket: int) -> None:
        """Forget a finished request's record (its Ticket can no longer be
        polled or waited on; the result buffer stays the caller's)."""
        L.call("blest_server_release", self._h, ticket)

    def drain(self, timeout_s: float = 600.0) -> None:
        L.call("blest_server_drain", self._h, timeout_s)

    def stats(self) -> dict:
        st = L.ServerStats()
        L.call("blest_server_stats_get", self._h, C.byref(st))
        return {k: getattr(st, k) for k, _ in L.ServerStats._fields_}
