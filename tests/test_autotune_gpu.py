"""Autotuner: picks a configuration from the timed table, caches it per
graph shape, and the tuned parameters give the oracle's levels."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import Csc, Graph
from blest_b200.autotune import tune_bfs, tune_mbfs
from graphs import prepared

pytestmark = pytest.mark.gpu


def test_tune_bfs_and_mbfs(tmp_path, gpu):
    csc, bvss, csr = prepared(Csc.rmat(13, 16, seed=4, permute_seed=3), "jaccard", 1024)
    g = Graph(bvss, csr)
    src = csc.sample_sources(8, seed=1)
    cache = str(tmp_path / "tune.json")
    space = {"blocks_per_sm": [1, 2], "alpha": [4.0, 14.0], "beta": [24.0], "slice_test": ["cuda_core", "mma"]}
    p, table = tune_bfs(g, src, space=space, cache=cache)
    assert len(table) == 8 and table[0]["seconds"] <= table[-1]["seconds"]
    for s in src[:3]:
        lv, _, _ = g.bfs(int(s), params=p)
        np.testing.assert_array_equal(lv, O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, int(s)))
    p2, table2 = tune_bfs(g, src, space=space, cache=cache)  # from the cache
    assert table2 == table and p2.blocks_per_sm == p.blocks_per_sm
    best, mtable = tune_mbfs(g, src, cache=cache)
    assert best["group_width"] in (32, 64, 128) and len(mtable) == 18
