"""The oracle checked against itself and the reference's fixtures (CPU).

The serial BVSS restatement of the reference's push step must agree with a
plain queue BFS on the CSC it was built from; CC fixpoints likewise; the
OpenMP CPU baseline must agree with both. Pins against the reference's BVSS
kernels run on a B200 live in tests/golden/ref_gpu_*.npz (see
tests/golden/make_golden_gpu.py) and are checked here when present.
"""
import numpy as np
import pytest

import oracle as O
from blest_b200 import Bvss, Csc
from conftest import GOLDEN


def _sources(n, k, seed):
    return np.random.default_rng(seed).choice(n, size=min(k, n), replace=False)


def test_bvss_restatement_equals_csc_bfs(host_golden):
    g = host_golden
    n = int(g["n"])
    arrays = {k: g[k] for k in ("slice_set_ptrs", "real_ptrs", "row_ids", "masks")}
    for s in _sources(n, 6, 1):
        a = O.bfs_csc(n, g["reordered_col_ptrs"], g["reordered_rows"], int(s))
        b = O.bfs_bvss(n, arrays, int(s))
        np.testing.assert_array_equal(a, b)


def test_cc_restatement_equals_csc_fixpoint(host_golden):
    g = host_golden
    n = int(g["n"])
    arrays = {k: g[k] for k in ("slice_set_ptrs", "real_ptrs", "row_ids", "masks")}
    a = O.cc_csc(n, g["reordered_col_ptrs"], g["reordered_rows"])
    b = O.cc_bvss(n, arrays)
    np.testing.assert_array_equal(a, b)
    c, _ = O.cc_omp(n, g["reordered_col_ptrs"], g["reordered_rows"], threads=4)
    np.testing.assert_array_equal(a, c)


def test_bfs_levels_are_hop_distances():
    # path 0-1-2-3 plus isolated 4, directed 5->0
    c = Csc.from_edges(6, [0, 1, 1, 2, 2, 3, 5], [1, 0, 2, 1, 3, 2, 0])
    lv = O.bfs_csc(6, c.col_ptrs, c.rows, 0)
    np.testing.assert_array_equal(lv, [0, 1, 2, 3, O.UNREACHED, O.UNREACHED])
    lv = O.bfs_csc(6, c.col_ptrs, c.rows, 5)
    np.testing.assert_array_equal(lv, [1, 2, 3, 4, O.UNREACHED, 0])
    lab = O.cc_csc(6, c.col_ptrs, c.rows)
    np.testing.assert_array_equal(lab, [0, 0, 0, 0, 4, 5])


@pytest.mark.parametrize("make", [lambda: Csc.rmat(12, 16, seed=2, permute_seed=1),
                                  lambda: Csc.grid(60, 50, 0.05, 0.002, seed=4),
                                  lambda: Csc.er(3000, 9000, seed=3)])
def test_omp_baseline_matches(make):
    c = make()
    t = c.transpose()
    for s in _sources(c.n, 4, 7):
        ref = O.bfs_csc(c.n, c.col_ptrs, c.rows, int(s))
        got, used = O.bfs_omp(c.n, c.col_ptrs, c.rows, t.col_ptrs, t.rows, int(s), threads=4)
        assert used == 4
        np.testing.assert_array_equal(got, ref)


def test_parent_checker_rejects_planted_mistakes():
    c = Csc.grid(20, 20, 0.0, 0.0, seed=1)
    n = c.n
    lv = O.bfs_csc(n, c.col_ptrs, c.rows, 0)
    # a valid parent array built on the CPU
    par = np.full(n, O.UNREACHED, dtype=np.uint32)
    par[0] = 0
    cp, rw = c.col_ptrs, c.rows
    for u in range(n):
        for v in rw[cp[u]:cp[u + 1]]:
            if lv[v] == lv[u] + 1 and par[v] == O.UNREACHED:
                par[v] = u
    assert O.check_parents(n, cp, rw, 0, lv, par) == 0
    bad = par.copy()
    bad[45] = 0  # not a neighbour of 45
    assert O.check_parents(n, cp, rw, 0, lv, bad) == 46
    bad = par.copy()
    bad[0] = 1
    assert O.check_parents(n, cp, rw, 0, lv, bad) == 1


def test_canonical_labels():
    lab = np.array([7, 7, 3, 3, 9], dtype=np.uint32)
    np.testing.assert_array_equal(O.canonical_min_labels(lab), [0, 0, 2, 2, 4])


GPU_PINS = sorted(GOLDEN.glob("ref_gpu_*.npz"))


@pytest.mark.skipif(not GPU_PINS, reason="no reference GPU fixtures committed")
@pytest.mark.parametrize("path", GPU_PINS, ids=lambda p: p.stem)
def test_oracle_pinned_to_reference_kernels(path):
    """Levels/labels the reference's BVSS kernels produced on a B200 equal the oracle's."""
    f = dict(np.load(path))
    h = dict(np.load(GOLDEN / f"host_{str(f['host'])}.npz"))
    n = int(h["n"])
    for s, lv in zip(f["sources"], f["levels"]):
        np.testing.assert_array_equal(O.bfs_csc(n, h["reordered_col_ptrs"], h["reordered_rows"], int(s)), lv)
    if "cc_raw" in f:
        np.testing.assert_array_equal(O.cc_csc(n, h["reordered_col_ptrs"], h["reordered_rows"]), f["cc_raw"])


@pytest.mark.parametrize("kind", ["rmat", "rmat_perm", "grid", "grid_perm", "er"])
def test_oracle_generator_equals_the_library(kind):
    """The reference arm of the benchmark builds its inputs with the oracle's
    generator; they must be the library's graphs byte for byte."""
    from blest_b200 import Csc
    if kind.startswith("rmat"):
        ps = 7 if kind == "rmat_perm" else 0
        n, cp, rw = O.gen_rmat(11, 12, 0.57, 0.19, 0.19, 9, ps)
        c = Csc.rmat(11, 12, 0.57, 0.19, 0.19, seed=9, permute_seed=ps)
    elif kind.startswith("grid"):
        ps = 3 if kind == "grid_perm" else 0
        n, cp, rw = O.gen_grid(61, 29, 0.05, 0.01, 4, ps)
        c = Csc.grid(61, 29, 0.05, 0.01, seed=4, permute_seed=ps)
    else:
        n, cp, rw = O.gen_er(3001, 20000, 5, 0)
        c = Csc.er(3001, 20000, seed=5)
    assert n == c.n
    np.testing.assert_array_equal(cp, c.col_ptrs)
    np.testing.assert_array_equal(rw, c.rows)
    np.testing.assert_array_equal(O.sample_sources(n, cp, 40, 11), c.sample_sources(40, 11))


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
def test_reference_upload_bytes_follow_its_arrays():
    """The reference arm's e2e byte count: what the stock hostCode copies to
    the device per call, from the sizes of the reference's own arrays."""
    n, cp, rw = O.gen_rmat(10, 8, seed=2, permute_seed=3)
    g = O.RefGraph.from_csc(n, cp, rw)
    g.reorder("jaccard", 256)
    g.build_bvss(full_padding=False)
    a = g.bvss()
    bvss = sum(a[k].nbytes for k in ("slice_set_ptrs", "virtual_to_real", "real_ptrs", "row_ids", "masks"))
    nnz = int(cp[-1])
    assert g.upload_bytes("bfs", nnz) == bvss + 4 * (n + 1) + 4 * nnz
    assert g.upload_bytes("cc", nnz) == bvss + 4 * n + 4 * a["virtual_to_real"].size
