"""The benchmark's first configuration at its full size, every source:
RMAT scale 16 (edge factor 16, a/b/c = .57/.19/.19, seeded id
permutation), Jaccard window 65536, 64 seeded sources sampled among
vertices of degree >= 1 (as bench.py builds it). Levels must equal the
oracle's and those of the reference's own BVSSBFSKernel::hostCode on the
same BVSS, and parents must form valid BFS trees."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import Bvss, Csc, Graph, bfs_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat16(gpu):
    csc = Csc.rmat(16, 16, 0.57, 0.19, 0.19, seed=1, permute_seed=1)
    src = csc.sample_sources(64, 1)
    inv = np.asarray(csc.reorder("jaccard", window=65536))
    bvss = Bvss.build(csc)
    return csc, bvss, Graph(bvss, csc), inv[src]


@pytest.mark.parametrize("direction", ["auto", "push"])
def test_all_64_sources_match_the_oracle(rmat16, direction):
    csc, bvss, g, sources = rmat16
    assert len(sources) == 64
    p = bfs_params(direction)
    for s in sources:
        lv, par, _ = g.bfs(int(s), parents=True, params=p)
        np.testing.assert_array_equal(lv, O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, int(s)), err_msg=f"source {s}")
        assert O.check_parents(csc.n, csc.col_ptrs, csc.rows, int(s), lv, par) == 0


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
def test_all_64_sources_match_the_reference_kernels(rmat16):
    csc, bvss, g, sources = rmat16
    ref = O.RefGraph.from_bvss(csc.n, bvss.arrays(), bvss.full_padding, bvss.update_divergence,
                               csc.col_ptrs, csc.rows)
    for s in sources:
        want, _, tl, nv = ref.bfs(int(s), csc.n)
        lv, _, st = g.bfs(int(s))
        np.testing.assert_array_equal(lv, want, err_msg=f"source {s}")
        assert (st.total_levels, st.no_visited) == (tl, nv)
