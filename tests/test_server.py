"""Query server: scheduling logic on CPU (dry-run mode) and, on the GPU,
results identical alone and in a concurrent mix."""
import threading
import time

import numpy as np
import pytest

from blest_b200 import BlestError
from blest_b200.server import Server


def test_dry_run_coalesces_bfs_and_shares_cc():
    srv = Server(lanes=1, max_batch=128, dry_run=True)
    g0 = srv.add_virtual_graph(1000)
    g1 = srv.add_virtual_graph(5000)
    # one lane: while the first job is being formed the others queue up
    tickets = [srv.submit_bfs(g0, i) for i in range(300)]
    tickets += [srv.submit_cc(g1) for _ in range(5)]
    tickets += [srv.submit_bfs(g1, i) for i in range(3)]
    srv.drain(30)
    infos = [t.info() for t in tickets]
    assert all(i.status == 0 for i in infos)
    bfs0 = [i.batch_size for i in infos[:300]]
    assert max(bfs0) <= 128 and sum(1 for b in bfs0 if b > 1) > 0
    cc = [i.batch_size for i in infos[300:305]]
    assert sum(1.0 / b for b in cc) < 5  # CC requests pending together shared runs
    # batch size recorded in out[0] by the dry executor
    assert all(int(t.out[0]) == i.batch_size for t, i in zip(tickets, infos))
    st = srv.stats()
    assert st["completed"] == 308 and st["rejected"] == 0
    assert st["jobs"] < 308
    assert st["p99_latency_s"] >= st["p50_latency_s"] >= 0


def test_dry_run_admission_shrinks_batches_and_refuses_the_impossible():
    n = 1 << 20
    # a 2-source batch needs 3*n*4 (state) + 2*4*n (levels) bytes = 20 MiB
    srv = Server(lanes=2, max_batch=128, memory_budget=21 << 20, dry_run=True)
    g = srv.add_virtual_graph(n)
    ts = [srv.submit_bfs(g, i) for i in range(64)]
    srv.drain(30)
    infos = [t.info() for t in ts]
    assert all(i.status == 0 for i in infos)
    assert max(i.batch_size for i in infos) <= 2
    st = srv.stats()
    assert st["peak_reserved_bytes"] <= 21 << 20
    # budget 0 bytes beyond resident: single BFS needs no scratch, batches cannot form
    srv2 = Server(lanes=1, memory_budget=1, dry_run=True)
    g2 = srv2.add_virtual_graph(n)
    ts2 = [srv2.submit_bfs(g2, i) for i in range(10)]
    srv2.drain(30)
    assert all(t.info().batch_size == 1 for t in ts2)


def test_dry_run_validation_and_threads():
    srv = Server(lanes=3, dry_run=True)
    g = srv.add_virtual_graph(100)
    with pytest.raises(BlestError):
        srv.submit_bfs(g, 100)  # source out of range
    with pytest.raises(BlestError):
        srv.submit_bfs(7, 0)  # unknown graph
    out = []

    def client(seed):
        rng = np.random.default_rng(seed)
        for _ in range(200):
            out.append(srv.submit_bfs(g, int(rng.integers(0, 100))))
            if rng.random() < 0.1:
                time.sleep(0.0005)

    th = [threading.Thread(target=client, args=(i,)) for i in range(4)]
    [t.start() for t in th]
    [t.join() for t in th]
    srv.drain(30)
    assert srv.stats()["completed"] == 800
    assert all(t.done() for t in out)


def test_dry_run_completion_queue_release_and_kind_stats():
    srv = Server(lanes=2, max_batch=16, dry_run=True, completion_queue=True)
    g = srv.add_virtual_graph(1000)
    ts = [srv.submit_bfs(g, i) for i in range(50)] + [srv.submit_cc(g) for _ in range(4)]
    seen = {}
    while len(seen) < len(ts):
        got = srv.next_done(30)
        assert got is not None
        tid, info = got
        assert tid not in seen and info.status == 0
        seen[tid] = info
        srv.release(tid)
    assert sorted(seen) == sorted(t.id for t in ts)
    # completion order: done times never go backwards
    done = [i.done_s for i in seen.values()]
    assert done == sorted(done)
    assert srv.next_done(0.01) is None  # nothing left: times out
    with pytest.raises(BlestError):
        srv.release(ts[0].id)  # already released: unknown ticket
    st = srv.stats()
    assert st["jobs"] == st["jobs_bfs"] + st["jobs_mbfs"] + st["jobs_cc"]
    assert st["jobs_bfs"] + st["requests_mbfs"] == 50 and st["requests_cc"] == 4
    assert st["jobs_mbfs"] >= 1 and st["busy_mbfs_s"] > 0
    # without a completion queue, next_done is refused
    srv2 = Server(lanes=1, dry_run=True)
    with pytest.raises(BlestError):
        srv2.next_done(0.01)


@pytest.mark.parametrize("always", [False, True])
def test_dry_run_adaptive_policy_runs_small_groups_alone(always):
    """Dry-run jobs take 1 ms alone and 20 ms batched. Once both are
    measured, the adaptive policy runs a few pending requests one by one
    (3 ms < 20 ms, with room for a loaded machine's oversleeping) but still
    batches forty (40 ms > 20 ms); BLEST_BATCH_ALWAYS batches both."""
    srv = Server(lanes=1, max_batch=128, dry_run=True, always_batch=always)
    g = srv.add_virtual_graph(1000)
    # a lone request, then ten at once (whatever the scheduler takes first,
    # the rest queue behind a 1 ms job and run as a batch): both estimates
    lone = srv.submit_bfs(g, 0)
    srv.drain(30)
    boot = [srv.submit_bfs(g, i) for i in range(10)]
    srv.drain(30)
    assert lone.info().batch_size == 1 and max(t.info().batch_size for t in boot) > 1
    small = []
    for _ in range(4):  # three at a time
        small += [srv.submit_bfs(g, i) for i in range(3)]
        srv.drain(30)
    big = [srv.submit_bfs(g, i) for i in range(41)]
    srv.drain(30)
    st = srv.stats()
    if always:
        assert st["unbatched_requests"] == 0
        assert max(t.info().batch_size for t in small) >= 2
    else:
        assert st["unbatched_requests"] >= 4
        assert all(t.info().batch_size == 1 for t in small)
    assert max(t.info().batch_size for t in big) >= 21
    with pytest.raises(BlestError):
        import ctypes as C
        from blest_b200 import _lib as L
        bad = L.ServerParams(0, 1, 0, 0, 1, 0, 7)
        L.call("blest_server_create", C.byref(bad), C.byref(C.c_void_p()))


@pytest.mark.gpu
def test_results_equal_alone_and_in_the_mix(gpu):
    import oracle as O
    from blest_b200 import Csc, Graph
    from graphs import prepared
    graphs = []
    for make in (lambda: Csc.rmat(14, 16, seed=1, permute_seed=2), lambda: Csc.grid(90, 70, 0.05, 0.01, seed=3),
                 lambda: Csc.er(6000, 30000, seed=5)):
        csc, bvss, csr = prepared(make(), "auto", 4096)
        graphs.append((csc, Graph(bvss, csr)))
    srv = Server(lanes=4, max_batch=64)
    gids = [srv.add_graph(g) for _, g in graphs]
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(400):
        gi = int(rng.integers(0, len(graphs)))
        if rng.random() < 0.2:
            reqs.append((gi, "cc", None, srv.submit_cc(gids[gi])))
        else:
            s = int(rng.integers(0, graphs[gi][0].n))
            reqs.append((gi, "bfs", s, srv.submit_bfs(gids[gi], s)))
        if rng.random() < 0.05:
            time.sleep(0.001)
    srv.drain(120)
    batched = 0
    for gi, kind, s, t in reqs:
        csc, g = graphs[gi]
        info = t.info()
        assert info.status == 0
        batched += info.batch_size > 1
        if kind == "bfs":
            alone, _, _ = g.bfs(s)
            np.testing.assert_array_equal(t.out, alone)
            np.testing.assert_array_equal(t.out, O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, s))
        else:
            alone, _ = g.cc()
            np.testing.assert_array_equal(t.out, alone)
    assert batched > 0  # some requests were coalesced
    st = srv.stats()
    assert st["completed"] == 400 and st["p99_latency_s"] > 0
    srv.close()


@pytest.mark.gpu
def test_device_results_equal_host_results(gpu):
    """Results written to device buffers (for a consumer on the GPU) equal
    the oracle's, alone and coalesced, for BFS and CC."""
    import torch
    import oracle as O
    from blest_b200 import Csc, Graph
    from graphs import prepared
    csc, bvss, csr = prepared(Csc.rmat(13, 16, seed=4, permute_seed=1), "jaccard", 4096)
    g = Graph(bvss, csr)
    srv = Server(lanes=2, max_batch=32)
    gid = srv.add_graph(g)
    srcs = [int(x) for x in csc.sample_sources(40, seed=3)]
    outs = [torch.empty(csc.n, dtype=torch.int32, device="cuda") for _ in srcs]
    tickets = [srv.submit_bfs(gid, s, out=o) for s, o in zip(srcs, outs)]
    cc_out = torch.empty(csc.n, dtype=torch.int32, device="cuda")
    tc = srv.submit_cc(gid, out=cc_out)
    srv.drain(60)
    batched = 0
    for s, o, t in zip(srcs, outs, tickets):
        assert t.info().status == 0
        batched += t.info().batch_size > 1
        np.testing.assert_array_equal(o.cpu().numpy().view(np.uint32), O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, s))
    assert batched > 0
    assert tc.info().status == 0
    np.testing.assert_array_equal(cc_out.cpu().numpy().view(np.uint32), O.cc_csc(csc.n, csc.col_ptrs, csc.rows))
    srv.close()


@pytest.mark.gpu
def test_batch_with_host_and_device_results(gpu):
    """One coalesced batch whose results go partly to device buffers
    (written by the kernel straight into them) and partly to host buffers
    (staged, then copied): every result equals the oracle's; finished
    tickets come back through the completion queue."""
    import torch
    import oracle as O
    from blest_b200 import Csc, Graph
    from graphs import prepared
    csc, bvss, csr = prepared(Csc.er(3001, 12000, seed=6), "rcm", 4096)
    g = Graph(bvss, csr)
    srv = Server(lanes=1, max_batch=128, completion_queue=True)
    gid = srv.add_graph(g)
    srcs = [int(x) for x in csc.sample_sources(70, seed=5)]
    # a first request occupies the lane while the rest queue up into one batch
    first = srv.submit_cc(gid)
    outs, tickets = [], []
    for i, s in enumerate(srcs):
        o = torch.empty(csc.n, dtype=torch.int32, device="cuda") if i % 3 else np.empty(csc.n, dtype=np.uint32)
        outs.append(o)
        tickets.append(srv.submit_bfs(gid, s, out=o))
    ids = set()
    for _ in range(len(srcs) + 1):
        got = srv.next_done(60)
        assert got is not None and got[1].status == 0
        ids.add(got[0])
    assert ids == {t.id for t in tickets} | {first.id}
    assert max(t.info().batch_size for t in tickets) > 1
    for s, o in zip(srcs, outs):
        got = o.cpu().numpy().view(np.uint32) if isinstance(o, torch.Tensor) else o
        np.testing.assert_array_equal(got, O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, s))
    st = srv.stats()
    assert st["requests_mbfs"] + st["jobs_bfs"] == len(srcs)
    # a host buffer passed as device memory is refused at submission, before
    # it could fail the batch it would join
    import ctypes as C
    from blest_b200 import _lib as L
    host = np.empty(csc.n, dtype=np.uint32)
    with pytest.raises(BlestError):
        L.call("blest_server_submit_ex", srv._h, gid, L.QUERY_BFS, srcs[0], host.ctypes.data, L.MEM_DEVICE,
               C.byref(L.u64()))
    srv.close()


@pytest.mark.gpu
def test_request_that_never_fits_is_refused(gpu):
    from blest_b200 import Csc, Graph
    from graphs import prepared
    csc, bvss, csr = prepared(Csc.rmat(12, 8, seed=1, permute_seed=1), "jaccard", 1024)
    g = Graph(bvss, csr)
    srv = Server(lanes=1, max_batch=128, memory_budget=1)
    gid = srv.add_graph(g)
    ts = [srv.submit_bfs(gid, i) for i in range(40)]
    srv.drain(60)
    # batches cannot be admitted; single-source queries need no extra scratch
    assert all(t.info().status == 0 and t.info().batch_size == 1 for t in ts)
    srv.close()


def test_dry_run_graphs_added_while_jobs_run():
    """Adding graphs (which grows the server's graph and workspace tables)
    while other jobs run leaves every request served."""
    srv = Server(lanes=3, max_batch=16, dry_run=True)
    g0 = srv.add_virtual_graph(500)
    tickets = []
    stop = threading.Event()

    def client():
        i = 0
        while not stop.is_set():
            tickets.append(srv.submit_bfs(g0, i % 500))
            i += 1
            time.sleep(0.0002)

    th = threading.Thread(target=client)
    th.start()
    added = []
    for k in range(40):
        gid = srv.add_virtual_graph(100 + k)
        added.append(gid)
        tickets.append(srv.submit_cc(gid))
        tickets.append(srv.submit_bfs(gid, k % (100 + k)))
    stop.set()
    th.join()
    srv.drain(60)
    assert all(t.info().status == 0 for t in tickets)
    assert srv.stats()["completed"] == len(tickets)
