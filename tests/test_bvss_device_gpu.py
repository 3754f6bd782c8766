"""BVSS construction on the GPU: every array byte for byte as the host
builder writes it (which the host-layer tests pin to the reference's own
builder), on the reference-generated fixtures and on generated graphs with
ragged sizes, duplicates-free and directed inputs, both padding rules; and
a resident graph built from a CSC this way gives the oracle's levels."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import Bvss, Csc, Graph
from conftest import GOLDEN
from graphs import prepared, random_directed, path, star

pytestmark = pytest.mark.gpu

ARRAYS = ("slice_set_ptrs", "virtual_to_real", "real_ptrs", "row_ids", "masks")


def _same(a: Bvss, b: Bvss):
    va, vb = a.view(), b.view()
    for f in ("n", "no_real_slice_sets", "no_virtual_slice_sets", "no_slices", "no_padded_slices", "full_padding"):
        assert getattr(va, f) == getattr(vb, f), f
    assert va.update_divergence == vb.update_divergence  # the same double
    xa, xb = a.arrays(), b.arrays()
    for k in ARRAYS:
        np.testing.assert_array_equal(xa[k], xb[k], err_msg=k)


@pytest.mark.parametrize("path_", sorted(GOLDEN.glob("host_*.npz")), ids=lambda p: p.stem)
def test_device_build_equals_reference_fixtures(gpu, path_):
    h = dict(np.load(path_))
    n = int(h["n"])
    csc = Csc.from_arrays(n, h["reordered_col_ptrs"], h["reordered_rows"])
    got = Bvss.build_device(csc, full_padding=bool(h["full_padding"]))
    for k in ARRAYS:
        np.testing.assert_array_equal(got.arrays()[k], h[k], err_msg=k)
    assert got.view().update_divergence == float(h["update_divergence"])


CASES = [
    ("rmat14_jaccard", lambda: Csc.rmat(14, 16, seed=5, permute_seed=2), "jaccard"),
    ("rmat16_natural", lambda: Csc.rmat(16, 16, seed=8, permute_seed=3), "natural"),
    ("grid101x77_rcm", lambda: Csc.grid(101, 77, 0.05, 0.001, seed=3), "rcm"),
    ("er5001", lambda: Csc.er(5001, 40000, seed=4), "natural"),
    ("directed_300", lambda: random_directed(300, 1500, 3), "natural"),
    ("star257", lambda: star(257), "natural"),  # one rset with more than 128 distinct rows
    ("path1001", lambda: path(1001), "natural"),
    ("one_vertex", lambda: Csc.from_arrays(1, [0, 0], []), "natural"),
]


@pytest.mark.parametrize("full_padding", [False, True])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_device_build_equals_host_build(gpu, case, full_padding):
    _, make, order = case
    csc = make()
    csc.reorder(order, window=4096)
    _same(Bvss.build_device(csc, full_padding), Bvss.build(csc, full_padding))


def test_graph_from_csc_matches_the_oracle(gpu):
    csc, _, csr = prepared(Csc.rmat(15, 16, seed=12, permute_seed=4), "jaccard", 8192)
    g = Graph.from_csc(csc)  # symmetric: the CSC is the pull CSR
    for s in csc.sample_sources(4, seed=2):
        lv, par, _ = g.bfs(int(s), parents=True)
        np.testing.assert_array_equal(lv, O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, int(s)))
        assert O.check_parents(csc.n, csc.col_ptrs, csc.rows, int(s), lv, par) == 0
    lab, _ = g.cc()
    np.testing.assert_array_equal(lab, O.cc_csc(csc.n, csc.col_ptrs, csc.rows))
    d = random_directed(500, 3000, 9)
    d.reorder("natural")
    gd = Graph.from_csc(d, d.transpose())
    lv, _, _ = gd.bfs(7)
    np.testing.assert_array_equal(lv, O.bfs_csc(d.n, d.col_ptrs, d.rows, 7))
