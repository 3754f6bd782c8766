"""Cache files interchange with the reference in both directions: the
reference's own writers (CSC::saveToBinary, CSC::saveOrderingToBinary,
BVSS::saveToBinary; DataStructures/CSC.cuh:225-266, :335-356,
DataStructures/BVSS.cuh:125-183, run through the harness) produce files
this library loads to the same arrays, and files this library writes load
in the reference's readers (CSC::constructFromBinary, CSC::orderFromBinary,
BVSS::constructFromBinary) to the same arrays."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import Bvss, Csc, load_ordering, save_ordering

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")

ARRAYS = ("slice_set_ptrs", "virtual_to_real", "real_ptrs", "row_ids", "masks")


@pytest.fixture(params=["rmat11_jaccard", "grid50x41_rcm"])
def graph(request):
    if request.param.startswith("rmat"):
        n, cp, rw = O.gen_rmat(11, 12, 0.57, 0.19, 0.19, 3, 4)
        mode = "jaccard"
    else:
        n, cp, rw = O.gen_grid(50, 41, 0.05, 0.01, 2, 0)
        mode = "rcm"
    return n, cp, rw, mode


def test_reference_files_load_here(tmp_path, graph):
    n, cp, rw, mode = graph
    ref = O.RefGraph.from_csc(n, cp, rw)
    ref.save_csc(tmp_path / "g_csc.bin")
    inv = ref.reorder(mode, 64)
    ref.save_ordering(tmp_path / "g_ordering.bin", inv)
    ref.build_bvss(not ref.is_social())
    ref.save_bvss(tmp_path / "g_bvss.bin")

    c = Csc.load_bin(str(tmp_path / "g_csc.bin"))
    assert c.n == n and c.is_social == ref.is_social()
    np.testing.assert_array_equal(c.col_ptrs, cp)
    np.testing.assert_array_equal(c.rows, rw)
    np.testing.assert_array_equal(load_ordering(str(tmp_path / "g_ordering.bin"), n), inv)
    b = Bvss.load_bin(str(tmp_path / "g_bvss.bin"))
    want = ref.bvss()
    for k in ARRAYS:
        np.testing.assert_array_equal(b.arrays()[k], want[k], err_msg=k)
    assert b.view().update_divergence == want["update_divergence"]


def test_files_written_here_load_in_the_reference(tmp_path, graph):
    n, cp, rw, mode = graph
    c = Csc.from_arrays(n, cp, rw)
    c.save_bin(str(tmp_path / "g_csc.bin"))
    r = O.RefGraph.load_csc(tmp_path / "g_csc.bin")
    rn, rnnz, rcp, rrw = r.csc()
    assert (rn, rnnz) == (n, len(rw)) and r.is_social() == c.is_social
    np.testing.assert_array_equal(rcp, cp)
    np.testing.assert_array_equal(rrw, rw)

    inv = np.asarray(c.reorder(mode, window=64), dtype=np.uint32)
    save_ordering(str(tmp_path / "g_ordering.bin"), inv)
    np.testing.assert_array_equal(r.load_ordering(tmp_path / "g_ordering.bin"), inv)
    # the reference applied it: its CSC is now ours
    _, _, rcp2, rrw2 = r.csc()
    np.testing.assert_array_equal(rcp2, c.col_ptrs)
    np.testing.assert_array_equal(rrw2, c.rows)

    b = Bvss.build(c)
    b.save_bin(str(tmp_path / "g_bvss.bin"))
    got = O.RefGraph.load_bvss(tmp_path / "g_bvss.bin").bvss()
    for k in ARRAYS:
        np.testing.assert_array_equal(got[k], b.arrays()[k], err_msg=k)
    assert got["update_divergence"] == b.view().update_divergence
