"""blest_bfs_noalloc: the allocation-free BFS entry point.

It serves callers that cannot call cudaMalloc (an application that hands
out all device memory from its own pool, a latency-critical path where
cudaMalloc/cudaFree could synchronise the device, a plugin that must not
grow memory per call). Such a caller already holds the graph and the output
buffers in its own device memory; here the test plays that caller, copies
the graph to the GPU itself, and calls the entry point through the C ABI.

Its levels must equal the oracle's and the regular entry point's
(blest_bfs) on consecutive calls that share the library's one scratch
array, including a graph at its vertex limit, a graph whose vertex count is
not a multiple of 8 or 32, and a smaller graph run right after a larger one
(whatever the larger left in the scratch must not leak into the result);
parents must form a valid BFS tree. Graphs above its vertex limit and
buffers that are not device memory are refused before any GPU work.
Integer results, so the tolerance is exact equality.
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
        np.testing.assert_array_equal(got, O.bfs_csc(n, csc.col_ptrs, csc.rows, s))
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


def _prepared(kind):
    if kind == "rmat20":
        csc = Csc.rmat(20, 16, seed=23, permute_seed=5)
        csc.reorder("jaccard", window=65536)
    else:
        csc = Csc.er(1001, 6000, seed=8)
        csc.reorder("rcm")
    return csc, Bvss.build(csc), csc.transpose()


def test_noalloc_at_its_limit_and_after_a_larger_graph(gpu):
    import torch
    big, small = _prepared("rmat20"), _prepared("er1001")
    assert big[0].n == L.NOALLOC_MAX_VERTICES and small[0].n % 8 != 0 and small[0].n % 32 != 0
    stream = torch.cuda.Stream()
    dev = {}
    for name, (csc, bvss, csr) in (("big", big), ("small", small)):
        view, keep = _device_graph(csc, bvss, csr)
        out = torch.empty(csc.n, dtype=torch.int32, device="cuda")
        par = torch.empty(csc.n, dtype=torch.int32, device="cuda")
        src = [int(s) for s in csc.sample_sources(2, seed=31)]
        dev[name] = (csc, view, keep, out, par, src)
    # big, small, big, small: each call reuses the scratch the previous
    # (differently sized) call left behind
    for name, i in (("big", 0), ("small", 0), ("big", 1), ("small", 1)):
        csc, view, keep, out, par, src = dev[name]
        s = src[i]
        st = L.BfsStats()
        L.call("blest_bfs_noalloc", C.byref(view), s, out.data_ptr(), par.data_ptr(), stream.cuda_stream,
               C.byref(st))
        got = out.cpu().numpy().view(np.uint32)
        want = O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, s)
        np.testing.assert_array_equal(got, want, err_msg=f"{name} source {s}")
        assert O.check_parents(csc.n, csc.col_ptrs, csc.rows, s, got, par.cpu().numpy().view(np.uint32)) == 0
        reached = want != O.UNREACHED
        assert st.no_visited == int(reached.sum())
        assert st.total_levels == int(want[reached].max()) + 1


def test_noalloc_refuses_host_buffers(gpu):
    csc, bvss, csr = _prepared("er1001")
    view, keep = _device_graph(csc, bvss, csr)
    host = np.empty(csc.n, dtype=np.uint32)
    # a host (unregistered) output buffer is refused before any launch
    with pytest.raises(BlestError) as e:
        L.call("blest_bfs_noalloc", C.byref(view), 0, host.ctypes.data, None, None, None)
    assert e.value.code == L.ERR_INVALID_ARG
    assert "not memory of the current device" in str(e.value)
