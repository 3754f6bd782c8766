"""Multi-source BFS on the B200: every source's level row equals the
single-source oracle BFS (bit-exact), for every group width, batch sizes
that do not fill a group, duplicate sources, and the many-graph batch."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import Graph
from graphs import golden_cases, prepared, small_cases

pytestmark = pytest.mark.gpu

CASES = small_cases() + golden_cases()


@pytest.fixture(params=CASES, ids=[c[0] for c in CASES])
def case(request, gpu):
    csc, bvss, csr = request.param[1]()
    return csc, bvss, csr, Graph(bvss, csr)


def _check(csc, sources, levels):
    for i, s in enumerate(sources):
        np.testing.assert_array_equal(levels[i], O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, int(s)),
                                      err_msg=f"source #{i} ({s})")


@pytest.mark.parametrize("width", [32, 64, 128])
def test_levels_equal_single_source(case, width):
    csc, bvss, csr, g = case
    rng = np.random.default_rng(width)
    k = min(csc.n, 77)
    sources = rng.choice(csc.n, size=k, replace=csc.n < k)
    levels, st = g.mbfs(sources, group_width=width)
    assert levels.shape == (k, csc.n)
    assert st.groups == (k + width - 1) // width
    _check(csc, sources, levels)


def test_duplicates_and_many_groups(gpu):
    from blest_b200 import Csc
    csc, bvss, csr = prepared(Csc.rmat(13, 16, seed=3, permute_seed=9), "jaccard", 1024)
    g = Graph(bvss, csr)
    rng = np.random.default_rng(5)
    sources = rng.choice(csc.n, size=300, replace=True)
    sources[:5] = sources[0]
    levels, st = g.mbfs(sources, group_width=128)
    assert st.groups == 3
    _check(csc, sources, levels)


def test_matches_single_source_kernel(gpu):
    from blest_b200 import Csc
    csc, bvss, csr = prepared(Csc.rmat(15, 16, seed=7, permute_seed=1), "jaccard", 4096)
    g = Graph(bvss, csr)
    sources = csc.sample_sources(130, seed=2)
    levels, _ = g.mbfs(sources)
    for i in (0, 64, 129):
        lv, _, _ = g.bfs(int(sources[i]))
        np.testing.assert_array_equal(levels[i], lv)


@pytest.mark.parametrize("name", ["path1000_fullpad", "grid101x77_rcm", "er5001_natural", "directed_300"])
def test_rows_per_source_buffers(name, gpu):
    """blest_mbfs_rows_ws: each source's levels land in its own device
    buffer (buffers allocated out of order, a partial second group, and on
    the 1000-level path the history overflows so rows also take the early
    partial writes); every row equals the oracle's and the source-major
    result."""
    import torch
    from blest_b200 import BlestError, Workspace
    csc, bvss, csr = dict(small_cases())[name]()
    g = Graph(bvss, csr)
    ws = Workspace(g)
    rng = np.random.default_rng(3)
    k = 150
    sources = rng.choice(csc.n, size=k, replace=csc.n < k)
    bufs = [torch.full((csc.n,), 7, dtype=torch.int32, device="cuda") for _ in range(k)]
    order = rng.permutation(k)  # row i is buffer order[i]: pointers in no memory order
    st = ws.mbfs_rows(sources, [bufs[j].data_ptr() for j in order], group_width=128)
    assert st.groups == 2
    torch.cuda.synchronize()
    ref, _ = g.mbfs(sources)
    for i, s in enumerate(sources):
        got = bufs[order[i]].cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, ref[i], err_msg=f"source #{i}")
        np.testing.assert_array_equal(got, O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, int(s)))
    # a host buffer among the rows is refused before any launch
    host = np.empty(csc.n, dtype=np.uint32)
    with pytest.raises(BlestError):
        ws.mbfs_rows(sources[:2], [bufs[0].data_ptr(), host.ctypes.data])
