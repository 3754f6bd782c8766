"""Asynchronous BFS calls on one workspace: every call's outcome is kept
(a ring of per-call records written by the kernel) and checked by
blest_workspace_sync, and host-output calls are pipelined (the copy of call
i overlaps the kernel of call i + 1) without changing any result."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import BlestError, Csc, Graph, Workspace
from blest_b200 import _lib as L
from graphs import prepared

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat(gpu):
    csc, bvss, csr = prepared(Csc.rmat(14, 16, seed=11, permute_seed=3), "jaccard", 4096)
    return csc, Graph(bvss, csr)


def test_pipelined_host_output_matches_the_oracle(rmat):
    import torch
    csc, g = rmat
    ws = Workspace(g)
    stream = torch.cuda.Stream()
    bufs = [torch.empty(csc.n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32) for _ in range(2)]
    sources = [int(s) for s in csc.sample_sources(9, seed=5)]
    want = {s: O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, s) for s in sources}
    # call i writes buffer i % 2; call i - 1 is settled after call i is
    # issued, so call i keeps running while call i - 1 is checked
    for i, s in enumerate(sources):
        ws.bfs_async(s, bufs[i % 2].ctypes.data, stream.cuda_stream, out_mem=L.MEM_HOST)
        if i:
            st = ws.sync_one()
            prev = sources[i - 1]
            assert st is not None and st.source_vertex == prev and st.time > 0
            np.testing.assert_array_equal(bufs[(i - 1) % 2], want[prev], err_msg=f"source {prev}")
    st = ws.sync_one()
    assert st.source_vertex == sources[-1]
    np.testing.assert_array_equal(bufs[(len(sources) - 1) % 2], want[sources[-1]])
    assert ws.sync_one() is None
    # sync settles all pending calls at once; stats are the last one's
    for i, s in enumerate(sources[:3]):
        ws.bfs_async(s, bufs[i % 2].ctypes.data if i < 2 else bufs[0].ctypes.data, stream.cuda_stream,
                     out_mem=L.MEM_HOST)
    assert ws.sync().source_vertex == sources[2]
    np.testing.assert_array_equal(bufs[1], want[sources[1]])
    np.testing.assert_array_equal(bufs[0], want[sources[2]])
    ws.close()


def test_every_async_call_is_checked(rmat):
    import torch
    csc, g = rmat
    ws = Workspace(g)
    stream = torch.cuda.Stream()
    out = torch.empty(csc.n, dtype=torch.int32, device="cuda")
    sources = [int(s) for s in csc.sample_sources(20, seed=6)]
    for s in sources:
        ws.bfs_async(s, out.data_ptr(), stream.cuda_stream)
    st = ws.sync()
    want = O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, sources[-1])
    reached = want != O.UNREACHED
    assert (st.source_vertex, st.no_visited, st.total_levels) == \
        (sources[-1], int(reached.sum()), int(want[reached].max()) + 1)
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), want)
    # a sync with nothing pending is a no-op; blocking calls still work
    ws.sync()
    lv = np.empty(csc.n, dtype=np.uint32)
    ws.bfs(sources[0], lv, stream.cuda_stream)
    np.testing.assert_array_equal(lv, O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, sources[0]))
    ws.close()


def test_more_async_calls_than_the_record_ring_are_reported(gpu):
    import torch
    csc, bvss, csr = prepared(Csc.rmat(8, 4, seed=2, permute_seed=1), "natural")
    g = Graph(bvss, csr)
    ws = Workspace(g)
    stream = torch.cuda.Stream()
    out = torch.empty(csc.n, dtype=torch.int32, device="cuda")
    for _ in range(1024 + 5):
        ws.bfs_async(0, out.data_ptr(), stream.cuda_stream)
    with pytest.raises(BlestError) as e:
        ws.sync()
    assert e.value.code == L.ERR_INVALID_ARG and "not checked" in str(e.value)
    ws.sync()  # settled: nothing pending any more
    ws.close()
