"""Multi-graph multi-source BFS in one persistent launch (blest_mbfs_plan_*,
blest_mbfs_batch): graphs of uneven sizes joined on the device, source slot
j shared by the j-th source of every graph. Every (graph, source) level row
must equal the single-source oracle BFS bit for bit, and the run is
replayed from a captured CUDA graph."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import Csc, Graph, MbfsPlan, mbfs_batch
from graphs import path, prepared, random_directed, star, two_cliques

pytestmark = pytest.mark.gpu


def _graphs():
    """(csc, Graph) pairs: ragged vertex counts (not multiples of 8 or 32),
    directed and undirected, high and low diameter."""
    out = []
    specs = [
        (path(45), "rcm"),
        (star(70), "auto"),
        (two_cliques(9), "auto"),
        (random_directed(301, 1500, 4), "auto"),
        (Csc.rmat(9, 8, seed=2, permute_seed=3), "jaccard"),
        (Csc.rmat(12, 16, seed=5, permute_seed=1), "jaccard"),
        (Csc.grid(37, 29, 0.05, 0.01, seed=3), "rcm"),
        (Csc.rmat(10, 4, seed=8, permute_seed=8), "jaccard"),
    ]
    for csc, order in specs:
        csc, bvss, csr = prepared(csc, order, 1024)
        out.append((csc, Graph(bvss, csr)))
    return out


@pytest.fixture(scope="module")
def graphs(gpu):
    return _graphs()


def _sources(csc, k, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, csc.n, size=k).astype(np.uint32)


def _check(csc, sources, levels):
    for i, s in enumerate(sources):
        np.testing.assert_array_equal(levels[i], O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, int(s)),
                                      err_msg=f"source #{i} ({s})")


def _plan(graphs, ks, width, seed=0):
    import torch
    outs, items, srcs = [], [], []
    for i, ((csc, g), k) in enumerate(zip(graphs, ks)):
        s = _sources(csc, k, seed + i)
        o = torch.full((max(k, 1), csc.n), 7, dtype=torch.int32, device="cuda")
        outs.append(o)
        srcs.append(s)
        items.append((g, s, o.data_ptr()))
    return MbfsPlan(items, group_width=width), outs, srcs


@pytest.mark.parametrize("width", [32, 64, 128])
def test_plan_matches_single_source(graphs, width):
    ks = [8, 1, 5, 40, 8, 130, 33, 0]
    plan, outs, srcs = _plan(graphs, ks, width)
    info = plan.info()
    assert info.items == len(graphs)
    assert info.n % 32 == 0 and info.n >= sum(c.n for c, _ in graphs)
    assert info.groups == (max(ks) + width - 1) // width
    assert info.captured == 1
    st = plan.run()
    assert st.groups == info.groups
    for (csc, _), k, o, s in zip(graphs, ks, outs, srcs):
        lv = o.cpu().numpy().view(np.uint32)
        if k == 0:
            assert (lv == 7).all()  # an item without sources is never written
            continue
        _check(csc, s, lv[:k])
    plan.close()


def test_plan_replay_and_new_sources(graphs):
    ks = [8] * len(graphs)
    plan, outs, srcs = _plan(graphs, ks, 32, seed=11)
    plan.run()
    first = [o.cpu().numpy().copy() for o in outs]
    plan.run()  # replay: identical
    for a, o in zip(first, outs):
        np.testing.assert_array_equal(a, o.cpu().numpy())
    new = [_sources(csc, 8, 100 + i) for i, (csc, _) in enumerate(graphs)]
    for i, s in enumerate(new):
        plan.set_sources(i, s)
    plan.launch()
    plan.sync()
    for (csc, _), o, s in zip(graphs, outs, new):
        _check(csc, s, o.cpu().numpy().view(np.uint32))
    with pytest.raises(Exception):
        plan.set_sources(0, np.full(8, graphs[0][0].n, dtype=np.uint32))  # out of range
    plan.close()


def test_batch_host_outputs(graphs):
    items, want = [], []
    for i, (csc, g) in enumerate(graphs):
        s = _sources(csc, 3 + i, 50 + i)
        lv = np.zeros((s.size, csc.n), dtype=np.uint32)
        items.append((g, s, lv))
        want.append((csc, s, lv))
    st = mbfs_batch(items, group_width=32)
    assert st.groups == 1
    for csc, s, lv in want:
        _check(csc, s, lv)


def test_single_graph_plan_equals_mbfs(graphs):
    import torch
    csc, g = graphs[5]
    s = _sources(csc, 100, 3)
    o = torch.empty((100, csc.n), dtype=torch.int32, device="cuda")
    plan = MbfsPlan([(g, s, o.data_ptr())], group_width=64)
    plan.run()
    lv, _ = g.mbfs(s, group_width=64)
    np.testing.assert_array_equal(o.cpu().numpy().view(np.uint32), lv)
    plan.close()
