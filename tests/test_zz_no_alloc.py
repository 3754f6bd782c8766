"""blest_bfs_noalloc: the allocation-free BFS entry point.

It serves callers that cannot call cudaMalloc (an application that hands
out all device memory from its own pool, a latency-critical path where
cudaMalloc/cudaFree could synchronise the device, a plugin that must not
grow memory per call). Such a caller already holds the graph and the output
buffers in its own device memory; here the test plays that caller, copies
the graph to the GPU itself, and calls the entry point through the C ABI.

Its levels and parents must equal the regular entry point's (blest_bfs) on
consecutive calls that share the library's one scratch array; graphs above
its vertex limit are refused before any GPU work. Integer results, so the
tolerance is exact equality.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from blest_b200 import BlestError, Bvss, Csc, Graph
from blest_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _to_device(a: np.ndarray):
    import torch
    a = np.ascontiguousarray(a)
    view = a.view(np.int64) if a.dtype == np.uint64 else a.view(np.int32)
    return torch.from_numpy(view.copy()).cuda()


def _device_graph(csc: Csc, bvss: Bvss, csr: Csc):
    arr = bvss.arrays()
    keep = {k: _to_device(v) for k, v in arr.items()}
    keep["csr_ptrs"] = _to_device(csr.col_ptrs)
    keep["csr_ids"] = _to_device(csr.rows)
    v = bvss.view()
    view = L.DeviceGraphView(csc.n, v.no_real_slice_sets, v.no_slices, csr.nnz,
                             keep["slice_set_ptrs"].data_ptr(), keep["real_ptrs"].data_ptr(),
                             keep["row_ids"].data_ptr(), keep["masks"].data_ptr(),
                             keep["csr_ptrs"].data_ptr(), keep["csr_ids"].data_ptr())
    return view, keep


def test_noalloc_equals_blest_bfs_on_consecutive_calls(gpu):
    import torch
    csc = Csc.rmat(15, 16, seed=21, permute_seed=4)
    csc.reorder("jaccard", window=4096)
    bvss = Bvss.build(csc)
    csr = csc.transpose()
    n = csc.n
    view, keep = _device_graph(csc, bvss, csr)
    levels = torch.empty(n, dtype=torch.int32, device="cuda")
    parents = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    g = Graph(bvss, csr)
    sources = [int(s) for s in csc.sample_sources(2, seed=9)]
    for s in (sources[0], sources[1], sources[0]):
        want, _, st_want = g.bfs(s)
        st = L.BfsStats()
        L.call("blest_bfs_noalloc", C.byref(view), s, levels.data_ptr(), parents.data_ptr(),
               stream.cuda_stream, C.byref(st))
        got = levels.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, want)
        par = parents.cpu().numpy().view(np.uint32)
        assert O.check_parents(n, csc.col_ptrs, csc.rows, s, got, par) == 0
        assert (st.no_visited, st.total_levels, st.reached_degree_sum) == \
            (st_want.no_visited, st_want.total_levels, st_want.reached_degree_sum)
    # without parents, on the default stream
    st = L.BfsStats()
    L.call("blest_bfs_noalloc", C.byref(view), sources[1], levels.data_ptr(), None, None, C.byref(st))
    want, _, _ = g.bfs(sources[1])
    np.testing.assert_array_equal(levels.cpu().numpy().view(np.uint32), want)


def test_noalloc_refuses_graphs_over_its_limit(gpu):
    n = L.NOALLOC_MAX_VERTICES + 1
    # Refused on the host before any pointer is used or any kernel runs.
    view = L.DeviceGraphView(n, (n + 7) // 8, 0, 0, 256, 256, 256, 256, 256, 256)
    with pytest.raises(BlestError) as e:
        L.call("blest_bfs_noalloc", C.byref(view), 0, 256, None, None, None)
    assert e.value.code == L.ERR_UNSUPPORTED
    assert "at most" in str(e.value)
