"""BFS parity on the B200 through the C ABI: levels bit-exact against the
oracle (and against the reference's own BVSS kernels on the same BVSS),
parents valid, for every direction policy and both slice tests."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import BlestError, Graph, bfs_params
from graphs import golden_cases, small_cases

pytestmark = pytest.mark.gpu

CASES = small_cases() + golden_cases()


def _sources(n, k=5, seed=0):
    rng = np.random.default_rng(seed)
    s = set(rng.choice(n, size=min(k, n), replace=False).tolist())
    s.add(0)
    s.add(n - 1)
    return sorted(s)


@pytest.fixture(params=CASES, ids=[c[0] for c in CASES])
def case(request, gpu):
    csc, bvss, csr = request.param[1]()
    return csc, bvss, csr, Graph(bvss, csr)


@pytest.mark.parametrize("direction", ["auto", "push", "pull"])
@pytest.mark.parametrize("test", ["cuda_core", "mma"])
def test_levels_bit_exact(case, direction, test):
    csc, bvss, csr, g = case
    p = bfs_params(direction, test)
    for s in _sources(csc.n):
        ref = O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, s)
        lv, par, st = g.bfs(s, parents=True, params=p)
        np.testing.assert_array_equal(lv, ref, err_msg=f"source {s}")
        assert O.check_parents(csc.n, csc.col_ptrs, csc.rows, s, lv, par) == 0
        reached = ref != O.UNREACHED
        assert st.no_visited == int(reached.sum())
        assert st.total_levels == int(ref[reached].max()) + 1
        assert st.reached_degree_sum == int(np.diff(csr.col_ptrs.astype(np.int64))[reached].sum())


def test_repeat_calls_are_identical(case):
    csc, bvss, csr, g = case
    s = _sources(csc.n)[-1]
    a, _, _ = g.bfs(s)
    b, _, _ = g.bfs(s)
    np.testing.assert_array_equal(a, b)


def test_invalid_source_rejected(case):
    csc, bvss, csr, g = case
    with pytest.raises(BlestError):
        g.bfs(csc.n)


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
def test_matches_reference_kernels(case):
    """Same BVSS into the reference's BVSSBFSKernel::hostCode: same levels."""
    csc, bvss, csr, g = case
    if csc.nnz == 0:
        pytest.skip("the reference kernels need at least one slice")
    ref = O.RefGraph.from_bvss(csc.n, bvss.arrays(), bvss.full_padding, bvss.update_divergence,
                               csr.col_ptrs, csr.rows)
    for s in _sources(csc.n, 3, 1):
        want, _, tl, nv = ref.bfs(s, csc.n)
        lv, _, st = g.bfs(s)
        np.testing.assert_array_equal(lv, want)
        assert st.total_levels == tl and st.no_visited == nv


def test_device_output_buffer(gpu):
    import torch
    from graphs import prepared
    from blest_b200 import Csc
    csc, bvss, csr = prepared(Csc.rmat(12, 16, seed=1, permute_seed=1), "jaccard", 1024)
    g = Graph(bvss, csr)
    out = torch.empty(csc.n, dtype=torch.int32, device="cuda")
    par = torch.empty(csc.n, dtype=torch.int32, device="cuda")
    st = g.bfs_device(7, out.data_ptr(), par.data_ptr())
    lv = out.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(lv, O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, 7))
    assert O.check_parents(csc.n, csc.col_ptrs, csc.rows, 7, lv, par.cpu().numpy().view(np.uint32)) == 0
    assert st.no_visited == int((lv != O.UNREACHED).sum())


def test_async_runs_then_sync_reports_the_last(gpu):
    """Asynchronous BFS calls queue no status copy; blest_workspace_sync
    waits and reports the last run's statistics."""
    import torch

    from blest_b200 import Csc, Workspace
    from graphs import prepared
    csc, bvss, csr = prepared(Csc.rmat(12, 16, seed=9, permute_seed=4), "jaccard", 1024)
    g = Graph(bvss, csr)
    ws = Workspace(g)
    out = torch.empty(csc.n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    sources = csc.sample_sources(6, seed=3)
    for s in sources:
        ws.bfs_async(int(s), out.data_ptr(), stream.cuda_stream)
    st = ws.sync()
    want = O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, int(sources[-1]))
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), want)
    reached = want != O.UNREACHED
    assert st.source_vertex == int(sources[-1])
    assert st.no_visited == int(reached.sum())
    assert st.total_levels == int(want[reached].max()) + 1
    ws.close()
