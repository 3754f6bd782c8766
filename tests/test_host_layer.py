"""Host layer (CSC classification, orderings, BVSS builder) against the
reference's own outputs stored in tests/golden/host_*.npz
(tests/golden/make_golden.py), plus format round trips and error paths."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import BlestError, Bvss, Csc, load_ordering, save_ordering


def _csc(g):
    return Csc.from_arrays(int(g["n"]), g["col_ptrs"], g["rows"])


def test_classification_matches_reference(host_golden):
    assert _csc(host_golden).is_social == bool(host_golden["is_social"])


def test_ordering_matches_reference(host_golden):
    g = host_golden
    c = _csc(g)
    mode = str(g["ordering"])
    inv = c.reorder(mode, window=int(g["window"]) or 65536)
    np.testing.assert_array_equal(inv, g["inverse_permutation"])
    np.testing.assert_array_equal(c.col_ptrs, g["reordered_col_ptrs"])
    np.testing.assert_array_equal(c.rows, g["reordered_rows"])


def test_bvss_matches_reference(host_golden):
    g = host_golden
    c = Csc.from_arrays(int(g["n"]), g["reordered_col_ptrs"], g["reordered_rows"])
    b = Bvss.build(c, full_padding=bool(g["full_padding"]))
    a = b.arrays()
    for k in ("slice_set_ptrs", "virtual_to_real", "real_ptrs", "row_ids", "masks"):
        np.testing.assert_array_equal(a[k], g[k], err_msg=k)
    assert b.update_divergence == float(g["update_divergence"])
    assert b.edge_check() == c.nnz  # the reference's "Check" line (BVSS.cuh:538)


def test_bvss_default_padding_follows_classification(host_golden):
    g = host_golden
    c = Csc.from_arrays(int(g["n"]), g["reordered_col_ptrs"], g["reordered_rows"])
    assert Bvss.build(c).full_padding == (not c.is_social)


def test_bvss_bin_roundtrip(tmp_path, host_golden):
    g = host_golden
    c = Csc.from_arrays(int(g["n"]), g["reordered_col_ptrs"], g["reordered_rows"])
    b = Bvss.build(c, full_padding=bool(g["full_padding"]))
    p = tmp_path / "g_bvss.bin"
    b.save_bin(str(p))
    b2 = Bvss.load_bin(str(p))
    for k, v in b.arrays().items():
        np.testing.assert_array_equal(b2.arrays()[k], v)
    assert b2.update_divergence == b.update_divergence
    # truncated file is rejected
    data = p.read_bytes()
    p.write_bytes(data[:-4])
    with pytest.raises(BlestError) as e:
        Bvss.load_bin(str(p))
    assert e.value.code == 8


def test_csc_bin_and_ordering_roundtrip(tmp_path):
    c = Csc.rmat(9, 8, seed=2, permute_seed=3)
    p = tmp_path / "x_csc.bin"
    c.save_bin(str(p))
    c2 = Csc.load_bin(str(p))
    np.testing.assert_array_equal(c2.col_ptrs, c.col_ptrs)
    np.testing.assert_array_equal(c2.rows, c.rows)
    assert c2.is_social == c.is_social
    # layout: n u32, nnz u32, isSocial u8, colPtrs, rows (CSC.cuh:225-266)
    raw = p.read_bytes()
    assert len(raw) == 9 + 4 * (c.n + 1) + 4 * c.nnz
    assert int.from_bytes(raw[:4], "little") == c.n
    inv = c.reorder("jaccard", window=64)
    q = tmp_path / "x_ordering.bin"
    save_ordering(str(q), inv)
    np.testing.assert_array_equal(load_ordering(str(q), c.n), inv)
    q.write_bytes(q.read_bytes()[:-4])
    with pytest.raises(BlestError):
        load_ordering(str(q), c.n)
    # corrupt CSC cache: row id out of range
    bad = bytearray(raw)
    bad[-4:] = (c.n + 5).to_bytes(4, "little")
    p.write_bytes(bytes(bad))
    with pytest.raises(BlestError):
        Csc.load_bin(str(p))


def test_mtx_reader_semantics(tmp_path):
    # "j i" lines: edge j -> i, self loops dropped, undirected adds reverse,
    # duplicates kept (CSC.cuh:98-185).
    p = tmp_path / "t.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern general\n% c\n4 4 5\n1 2\n2 3\n3 3\n4 1\n1 2\n")
    c = Csc.read_mtx(str(p), undirected=False, binary=True)
    assert c.n == 4 and c.nnz == 4
    np.testing.assert_array_equal(c.col_ptrs, [0, 2, 3, 3, 4])
    np.testing.assert_array_equal(c.rows, [1, 1, 2, 0])
    c = Csc.read_mtx(str(p), undirected=True, binary=True)
    assert c.nnz == 8
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 2\n2 1 0.5\n3 2 1.0\n")
    c = Csc.read_mtx(str(p))
    assert c.nnz == 4 and c.is_symmetric()
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n2 1 0.5\n")
    with pytest.raises(BlestError):
        Csc.read_mtx(str(p))
    with pytest.raises(BlestError):
        Csc.read_mtx(str(tmp_path / "missing.mtx"))


def test_generators_deterministic_and_clean():
    a = Csc.rmat(10, 16, seed=9, permute_seed=4)
    b = Csc.rmat(10, 16, seed=9, permute_seed=4)
    np.testing.assert_array_equal(a.rows, b.rows)
    c = Csc.rmat(10, 16, seed=10, permute_seed=4)
    assert not np.array_equal(a.rows, c.rows) or not np.array_equal(a.col_ptrs, c.col_ptrs)
    for g in (a, Csc.grid(30, 20, 0.05, 0.01, seed=3), Csc.er(500, 3000, seed=1)):
        assert g.is_symmetric()
        cp, rw = g.col_ptrs, g.rows
        cols = np.repeat(np.arange(g.n), np.diff(cp))
        assert not np.any(cols == rw), "self loop"
        for j in range(0, g.n, max(1, g.n // 50)):
            seg = rw[cp[j]:cp[j + 1]]
            assert np.all(np.diff(seg.astype(np.int64)) > 0), "unsorted or duplicate"
    gr = Csc.grid(16, 16, 0.0, 0.0, seed=1)
    assert gr.nnz == 2 * (2 * 16 * 15)


def test_sample_sources():
    g = Csc.rmat(10, 4, seed=1, permute_seed=1)
    s = g.sample_sources(64, seed=5)
    assert s.size == 64 and np.unique(s).size == 64
    assert np.all(g.degrees()[s] >= 1)
    np.testing.assert_array_equal(s, g.sample_sources(64, seed=5))


def test_permutation_check():
    c = Csc.rmat(6, 4, seed=1)
    with pytest.raises(BlestError):
        c.apply_permutation(np.zeros(c.n, dtype=np.uint32))


def test_bvss_from_arrays_rejects_bad_input(host_golden):
    g = host_golden
    a = {k: g[k].copy() for k in ("slice_set_ptrs", "virtual_to_real", "real_ptrs", "row_ids", "masks")}
    Bvss.from_arrays(int(g["n"]), **a)
    bad = {k: v.copy() for k, v in a.items()}
    nz = np.nonzero(bad["masks"] & 0xFF)[0]
    bad["row_ids"][4 * nz[0]] = int(g["n"]) + 3
    with pytest.raises(BlestError):
        Bvss.from_arrays(int(g["n"]), **bad)
    bad = {k: v.copy() for k, v in a.items()}
    bad["real_ptrs"][-1] += 1
    with pytest.raises(BlestError):
        Bvss.from_arrays(int(g["n"]), **bad)


def test_relabel_dense():
    from blest_b200 import relabel_dense
    lab = np.array([0, 0, 2, 2, 0, 5, 5], dtype=np.uint32)
    d, k = relabel_dense(lab)
    assert k == 3
    np.testing.assert_array_equal(d, [0, 0, 1, 1, 0, 2, 2])


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("make", [lambda: Csc.rmat(16, 16, seed=2, permute_seed=2),
                                  lambda: Csc.er(1 << 16, 16 << 15, seed=3),
                                  lambda: Csc.grid(300, 200, 0.3, 0.001, seed=3),
                                  lambda: Csc.er(1 << 18, 16 << 18, seed=4),
                                  lambda: Csc.rmat(17, 16, seed=6, permute_seed=3)],
                         ids=["rmat16", "er16", "grid300x200", "er18_deg32", "rmat17"])
def test_rcm_matches_reference_on_parallel_levels(make):
    """RCM orders big enough that levels run on the parallel paths (more
    than 2^16 edges per level: top-down claims, and bottom-up steps once the
    unreached vertices hold fewer edges than the level) equal the
    reference's sequential order, including the many small components of
    RMAT graphs."""
    c = make()
    want = O.RefGraph.from_csc(c.n, c.col_ptrs, c.rows).reorder("rcm")
    np.testing.assert_array_equal(c.reorder("rcm"), want)


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("make", [
    lambda: Csc.rmat(12, 8, seed=3, permute_seed=2),
    lambda: Csc.rmat(14, 16, seed=5, permute_seed=1),
    lambda: Csc.grid(60, 40, 0.05, 0.01, seed=2),
    lambda: Csc.er(2000, 1500, seed=7),  # isolated vertices
    lambda: Csc.from_edges(300, *zip(*[(i, (i * 7 + 3) % 300) for i in range(300)])),  # directed
], ids=["rmat12", "rmat14", "grid60x40", "er_isolated", "directed300"])
def test_gorder_matches_reference(make):
    """BLEST_ORDER_GORDER gives the permutation of the reference's
    CSC::gorder(8) (the vendored Gorder greedy, run through the harness)."""
    c = make()
    want = O.RefGraph.from_csc(c.n, c.col_ptrs, c.rows).reorder("gorder")
    got = c.reorder("gorder")
    np.testing.assert_array_equal(np.asarray(got), want)


def test_transpose_and_symmetry_check_on_directed_input():
    """The parallel transpose gives every transposed list in increasing
    column order (duplicates kept), as a sequential fill would; the parallel
    symmetry check finds a single missing reverse edge."""
    rng = np.random.default_rng(7)
    n = 3000
    src = rng.integers(0, n, 40000)
    dst = rng.integers(0, n, 40000)
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    ptrs = np.concatenate([[0], np.cumsum(np.bincount(src, minlength=n))]).astype(np.uint32)
    g = Csc.from_arrays(n, ptrs, dst.astype(np.uint32))
    t = g.transpose()
    cols = np.repeat(np.arange(n), np.diff(g.col_ptrs.astype(np.int64)))
    want = np.lexsort((cols, g.rows))
    np.testing.assert_array_equal(t.rows, cols[want])
    np.testing.assert_array_equal(t.col_ptrs, np.concatenate([[0], np.cumsum(np.bincount(g.rows, minlength=n))]))
    assert not g.is_symmetric()
    s = Csc.rmat(12, 8, seed=1, permute_seed=1)
    assert s.is_symmetric()
    # drop one reverse edge of the last column: asymmetric again
    cp, rw = s.col_ptrs.astype(np.int64), s.rows.copy()
    j = s.n - 1
    while cp[j + 1] == cp[j]:
        j -= 1
    keep = np.ones(rw.size, dtype=bool)
    keep[cp[j + 1] - 1] = False
    ptrs2 = cp.copy()
    ptrs2[j + 1:] -= 1
    a = Csc.from_arrays(s.n, ptrs2.astype(np.uint32), rw[keep])
    assert not a.is_symmetric()


def _mtx_expected(text: str, undirected: bool, binary: bool):
    """The reader's semantics restated: leading '%' lines skipped, then a
    whitespace token stream 'n n entries' and per entry 'j i [value]'; self
    loops dropped before the range check, duplicates kept, columns sorted."""
    lines = text.split("\n")
    k = 0
    while k < len(lines) and lines[k].startswith("%"):
        k += 1
    tok = "\n".join(lines[k:]).split()
    n, entries = int(tok[0]), int(tok[2])
    per = 2 if binary else 3
    cols = [[] for _ in range(n)]
    body = tok[3:]
    if len(body) < entries * per:
        return None
    for e in range(entries):
        j, i = int(body[e * per]), int(body[e * per + 1])
        if i == j:
            continue
        cols[j - 1].append(i - 1)
        if undirected:
            cols[i - 1].append(j - 1)
    ptr = np.concatenate([[0], np.cumsum([len(c) for c in cols])]).astype(np.uint32)
    rows = np.array([r for c in cols for r in sorted(c)], dtype=np.uint32)
    return ptr, rows


@pytest.mark.parametrize("seed", range(6))
def test_mtx_reader_token_stream_any_layout(tmp_path, seed):
    """The parallel reader cuts the file into per-thread chunks at token
    boundaries: entries split across lines or chunks, several entries on a
    line, tabs, CRLF, blank lines, self loops with out-of-range ids and
    trailing tokens all read as the sequential token stream does."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(3, 40))
    m = int(rng.integers(1, 300))
    binary = bool(seed % 2)
    undirected = seed % 3 == 0
    toks = []
    for _ in range(m):
        j, i = int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1))
        if rng.random() < 0.05:
            j = i = n + 7  # self loop out of range: dropped before the range check
        toks += [str(j), str(i)] + ([] if binary else [f"{rng.normal():.3e}"])
    seps = [" ", "\t", "\n", "\r\n", "  \n\n", " \t "]
    body = "".join(t + seps[int(rng.integers(0, len(seps)))] for t in toks)
    text = "%%MatrixMarket matrix coordinate x general\n% comment\n" + f"{n} {n} {m}\n" + body + "99 98\n"
    p = tmp_path / "g.mtx"
    p.write_bytes(text.encode())
    want = _mtx_expected(text, undirected, binary)
    c = Csc.read_mtx(str(p), undirected=undirected, binary=binary)
    np.testing.assert_array_equal(c.col_ptrs, want[0])
    np.testing.assert_array_equal(c.rows, want[1])


def test_mtx_reader_errors_follow_the_first_bad_entry(tmp_path):
    p = tmp_path / "e.mtx"
    head = "%%MatrixMarket matrix coordinate real general\n"
    # a value that is not a number
    p.write_text(head + "3 3 3\n1 2 0.5\n2 3 x\n3 1 1.0\n")
    with pytest.raises(BlestError, match="missing value"):
        Csc.read_mtx(str(p), undirected=False, binary=False)
    # out of range before a later truncation
    p.write_text(head + "3 3 3\n1 9 0.5\n2 3 1.0\n")
    with pytest.raises(BlestError, match="out of range"):
        Csc.read_mtx(str(p), undirected=False, binary=False)
    # truncated
    p.write_text(head + "3 3 3\n1 2 0.5\n2 3 1.0\n3\n")
    with pytest.raises(BlestError, match="truncated"):
        Csc.read_mtx(str(p), undirected=False, binary=False)
    p.write_text(head + "3 x 3\n")
    with pytest.raises(BlestError, match="size line"):
        Csc.read_mtx(str(p), undirected=False, binary=False)
