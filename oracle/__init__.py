"""CPU oracle for the BLEST B200 hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference legs may import this package; the product (blest_b200) never does.

- liboracle.so (oracle.c): serial BFS over the CSC, a serial restatement of
  the reference's BVSS push step, CC label-propagation fixpoints, parent
  validation, and the OpenMP direction-optimising CPU BFS baseline.
- _ref/libblest_ref.so (ref_harness.cu, built from the reference's own
  sources by oracle/Makefile): the reference's CSC orderings, BVSS builder
  and BVSS BFS/CC kernels behind a small C API. Present when the reference
  sources were available at build time (it travels as a built file).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libblest_ref.so"
UNREACHED = 0xFFFFFFFF

P32 = C.POINTER(C.c_uint32)
P64 = C.POINTER(C.c_uint64)


def build(ref: bool = True) -> None:
    """make -C oracle (liboracle.so; _ref/libblest_ref.so when the
    reference sources exist)."""
    target = "all" if ref else "liboracle.so"
    r = subprocess.run(["make", "-C", str(HERE), target], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


def _p32(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(P32)


def _p64(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(P64)


_olib = None


class OracleGraph(C.Structure):
    _fields_ = [("n", C.c_uint32), ("nnz", C.c_uint64), ("col_ptrs", P32), ("rows", P32)]


def olib():
    global _olib
    if _olib is None:
        if not ORACLE_SO.exists():
            build(ref=False)
        lib = C.CDLL(str(ORACLE_SO))
        lib.oracle_bfs_csc.argtypes = [C.c_uint32, P32, P32, C.c_uint32, P32]
        lib.oracle_bfs_bvss.argtypes = [C.c_uint32, C.c_uint32, P64, P32, P32, P32, C.c_uint32, P32]
        lib.oracle_cc_csc.argtypes = [C.c_uint32, P32, P32, P32]
        lib.oracle_cc_bvss.argtypes = [C.c_uint32, C.c_uint32, P64, P32, P32, P32, P32]
        lib.oracle_check_parents.argtypes = [C.c_uint32, P32, P32, C.c_uint32, P32, P32]
        lib.oracle_check_parents.restype = C.c_int64
        lib.oracle_bfs_omp.argtypes = [C.c_uint32, P32, P32, P32, P32, C.c_uint32, P32, C.c_int]
        lib.oracle_cc_omp.argtypes = [C.c_uint32, P32, P32, P32, C.c_int]
        lib.oracle_reached_degree_sum.argtypes = [C.c_uint32, P32, P32]
        lib.oracle_reached_degree_sum.restype = C.c_uint64
        for name, args in (("oracle_gen_rmat", [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                                C.c_uint64, C.c_uint64, C.POINTER(OracleGraph)]),
                           ("oracle_gen_grid", [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint64,
                                                C.c_uint64, C.POINTER(OracleGraph)]),
                           ("oracle_gen_er", [C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64,
                                              C.POINTER(OracleGraph)])):
            getattr(lib, name).argtypes = args
        lib.oracle_graph_free.argtypes = [C.POINTER(OracleGraph)]
        lib.oracle_graph_free.restype = None
        lib.oracle_sample_sources.argtypes = [C.c_uint32, P32, C.c_uint32, C.c_uint64, P32, P32]
        _olib = lib
    return _olib


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def bfs_csc(n, col_ptrs, rows, src) -> np.ndarray:
    cp, rw = _u32(col_ptrs), _u32(rows) if len(rows) else np.zeros(1, np.uint32)
    out = np.empty(n, dtype=np.uint32)
    assert olib().oracle_bfs_csc(n, _p32(cp), _p32(rw), src, _p32(out)) == 0
    return out


def bfs_bvss(n, arrays: dict, src) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    ssp = np.ascontiguousarray(arrays["slice_set_ptrs"], dtype=np.uint64)
    rp = _u32(arrays["real_ptrs"])
    ri = _u32(arrays["row_ids"]) if len(arrays["row_ids"]) else np.zeros(4, np.uint32)
    mk = _u32(arrays["masks"]) if len(arrays["masks"]) else np.zeros(1, np.uint32)
    rc = olib().oracle_bfs_bvss(n, rp.size - 1, _p64(ssp), _p32(rp), _p32(ri), _p32(mk), src, _p32(out))
    assert rc == 0, rc
    return out


def cc_csc(n, col_ptrs, rows) -> np.ndarray:
    cp, rw = _u32(col_ptrs), _u32(rows) if len(rows) else np.zeros(1, np.uint32)
    out = np.empty(n, dtype=np.uint32)
    assert olib().oracle_cc_csc(n, _p32(cp), _p32(rw), _p32(out)) == 0
    return out


def cc_bvss(n, arrays: dict) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    ssp = np.ascontiguousarray(arrays["slice_set_ptrs"], dtype=np.uint64)
    rp = _u32(arrays["real_ptrs"])
    ri = _u32(arrays["row_ids"]) if len(arrays["row_ids"]) else np.zeros(4, np.uint32)
    mk = _u32(arrays["masks"]) if len(arrays["masks"]) else np.zeros(1, np.uint32)
    assert olib().oracle_cc_bvss(n, rp.size - 1, _p64(ssp), _p32(rp), _p32(ri), _p32(mk), _p32(out)) == 0
    return out


def check_parents(n, col_ptrs, rows, src, levels, parents) -> int:
    cp, rw = _u32(col_ptrs), _u32(rows) if len(rows) else np.zeros(1, np.uint32)
    return int(olib().oracle_check_parents(n, _p32(cp), _p32(rw), src, _p32(_u32(levels)), _p32(_u32(parents))))


def bfs_omp(n, col_ptrs, rows, in_ptrs, in_ids, src, threads=0):
    cp, rw, ip, ii = _u32(col_ptrs), _u32(rows), _u32(in_ptrs), _u32(in_ids)
    out = np.empty(n, dtype=np.uint32)
    used = olib().oracle_bfs_omp(n, _p32(cp), _p32(rw), _p32(ip), _p32(ii), src, _p32(out), threads)
    assert used > 0
    return out, used


def cc_omp(n, col_ptrs, rows, threads=0):
    cp, rw = _u32(col_ptrs), _u32(rows)
    out = np.empty(n, dtype=np.uint32)
    used = olib().oracle_cc_omp(n, _p32(cp), _p32(rw), _p32(out), threads)
    return out, used


def _take_graph(fn, *args):
    g = OracleGraph()
    rc = fn(*args, C.byref(g))
    if rc != 0:
        raise RuntimeError(f"oracle graph generator failed ({rc})")
    try:
        cp = np.ctypeslib.as_array(g.col_ptrs, shape=(g.n + 1,)).copy()
        rw = np.ctypeslib.as_array(g.rows, shape=(max(g.nnz, 1),))[: g.nnz].copy()
    finally:
        olib().oracle_graph_free(C.byref(g))
    return g.n, cp, rw


def gen_rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=1, permute_seed=0):
    """(n, col_ptrs, rows) of the seeded RMAT graph blest_csc_generate_rmat makes."""
    return _take_graph(olib().oracle_gen_rmat, scale, edge_factor, a, b, c, seed, permute_seed)


def gen_grid(width, height, p_delete, shortcut_fraction, seed=1, permute_seed=0):
    return _take_graph(olib().oracle_gen_grid, width, height, p_delete, shortcut_fraction, seed, permute_seed)


def gen_er(n, m, seed=1, permute_seed=0):
    return _take_graph(olib().oracle_gen_er, n, m, seed, permute_seed)


def sample_sources(n, col_ptrs, k, seed) -> np.ndarray:
    out = np.empty(max(k, 1), dtype=np.uint32)
    cnt = C.c_uint32()
    assert olib().oracle_sample_sources(n, _p32(_u32(col_ptrs)), k, seed, _p32(out), C.byref(cnt)) == 0
    return out[: cnt.value].copy()


def reached_degree_sum(n, col_ptrs, levels) -> int:
    return int(olib().oracle_reached_degree_sum(n, _p32(_u32(col_ptrs)), _p32(_u32(levels))))


def canonical_min_labels(labels: np.ndarray) -> np.ndarray:
    """Relabel every vertex by the smallest vertex id carrying its label
    (makes any partition labelling comparable)."""
    labels = np.asarray(labels)
    n = labels.size
    first = np.full(int(labels.max()) + 1 if n else 1, np.iinfo(np.int64).max, dtype=np.int64)
    np.minimum.at(first, labels.astype(np.int64), np.arange(n, dtype=np.int64))
    return first[labels.astype(np.int64)].astype(np.uint32)


# ---------------------------------------------------------------- reference
_rlib = None


def ref_available() -> bool:
    return REF_SO.exists()


def rlib():
    global _rlib
    if _rlib is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference sources at build time)")
        lib = C.CDLL(str(REF_SO))
        vp = C.c_void_p
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_csc_create.argtypes = [C.c_uint32, P32, P32, C.POINTER(vp)]
        lib.ref_csc_is_social.argtypes = [vp, C.POINTER(C.c_int)]
        lib.ref_csc_reorder.argtypes = [vp, C.c_int, C.c_uint32, C.c_uint32, P32]
        lib.ref_csc_get.argtypes = [vp, P32, P32, C.POINTER(P32), C.POINTER(P32)]
        lib.ref_bvss_build.argtypes = [vp, C.c_int]
        lib.ref_bvss_get.argtypes = [vp, P32, P32, P32, P64, C.POINTER(C.c_double), C.POINTER(P64),
                                     C.POINTER(P32), C.POINTER(P32), C.POINTER(P32), C.POINTER(P32)]
        lib.ref_bvss_from_arrays.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_double, C.c_int,
                                             P64, P32, P32, P32, P32, C.c_uint32, P32, P32, C.POINTER(vp)]
        lib.ref_bfs_variant.argtypes = [vp, C.POINTER(C.c_int)]
        lib.ref_bfs.argtypes = [vp, C.c_uint32, P32, C.POINTER(C.c_double), P32, P32]
        lib.ref_cc.argtypes = [vp, P32, C.POINTER(C.c_double), P32]
        lib.ref_cc_raw.argtypes = [vp, P32, C.POINTER(C.c_double)]
        lib.ref_destroy.argtypes = [vp]
        lib.ref_csc_save.argtypes = [vp, C.c_char_p]
        lib.ref_csc_load.argtypes = [C.c_char_p, C.POINTER(vp)]
        lib.ref_ordering_save.argtypes = [vp, C.c_char_p, P32]
        lib.ref_ordering_load.argtypes = [vp, C.c_char_p, P32]
        lib.ref_bvss_save.argtypes = [vp, C.c_char_p]
        lib.ref_bvss_load.argtypes = [C.c_char_p, C.POINTER(vp)]
        _rlib = lib
    return _rlib


def _rcheck(rc):
    if rc != 0:
        raise RuntimeError("reference harness: " + rlib().ref_last_error().decode())


class RefGraph:
    """The reference's CSC/BVSS objects (oracle/_ref)."""

    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None):
            rlib().ref_destroy(self.h)
            self.h = None

    @classmethod
    def from_csc(cls, n, col_ptrs, rows) -> "RefGraph":
        h = C.c_void_p()
        cp, rw = _u32(col_ptrs), _u32(rows) if len(rows) else np.zeros(1, np.uint32)
        _rcheck(rlib().ref_csc_create(n, _p32(cp), _p32(rw), C.byref(h)))
        return cls(h)

    @classmethod
    def from_bvss(cls, n, arrays: dict, full_padding: bool, divergence: float, csr_ptrs, csr_ids) -> "RefGraph":
        h = C.c_void_p()
        ssp = np.ascontiguousarray(arrays["slice_set_ptrs"], dtype=np.uint64)
        v2r, rp = _u32(arrays["virtual_to_real"]), _u32(arrays["real_ptrs"])
        ri, mk = _u32(arrays["row_ids"]), _u32(arrays["masks"])
        cp, ci = _u32(csr_ptrs), _u32(csr_ids)
        _rcheck(rlib().ref_bvss_from_arrays(n, rp.size - 1, v2r.size, ri.size, divergence, int(full_padding),
                                            _p64(ssp), _p32(v2r), _p32(rp), _p32(ri), _p32(mk), ci.size,
                                            _p32(cp), _p32(ci), C.byref(h)))
        return cls(h)

    @classmethod
    def load_csc(cls, path) -> "RefGraph":
        """CSC::constructFromBinary of a _csc.bin file."""
        h = C.c_void_p()
        _rcheck(rlib().ref_csc_load(str(path).encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def load_bvss(cls, path) -> "RefGraph":
        """BVSS::constructFromBinary of a _bvss.bin file."""
        h = C.c_void_p()
        _rcheck(rlib().ref_bvss_load(str(path).encode(), C.byref(h)))
        return cls(h)

    def save_csc(self, path) -> None:
        _rcheck(rlib().ref_csc_save(self.h, str(path).encode()))

    def save_ordering(self, path, inv) -> None:
        _rcheck(rlib().ref_ordering_save(self.h, str(path).encode(), _p32(_u32(inv))))

    def load_ordering(self, path) -> np.ndarray:
        """CSC::orderFromBinary: read and apply; returns the permutation."""
        n = self.csc()[0]
        inv = np.empty(n, dtype=np.uint32)
        _rcheck(rlib().ref_ordering_load(self.h, str(path).encode(), _p32(inv)))
        return inv

    def save_bvss(self, path) -> None:
        _rcheck(rlib().ref_bvss_save(self.h, str(path).encode()))

    def is_social(self) -> bool:
        s = C.c_int()
        _rcheck(rlib().ref_csc_is_social(self.h, C.byref(s)))
        return bool(s.value)

    def reorder(self, mode: str, window: int = 65536, rand_seed: int = 1) -> np.ndarray:
        n, nnz, cp, rw = self.csc()
        inv = np.empty(n, dtype=np.uint32)
        m = {"natural": 1, "jaccard": 2, "rcm": 3, "gorder": 4}[mode]
        _rcheck(rlib().ref_csc_reorder(self.h, m, window, rand_seed, _p32(inv)))
        return inv

    def csc(self):
        n, nnz = C.c_uint32(), C.c_uint32()
        cp, rw = P32(), P32()
        _rcheck(rlib().ref_csc_get(self.h, C.byref(n), C.byref(nnz), C.byref(cp), C.byref(rw)))
        cpa = np.ctypeslib.as_array(cp, shape=(n.value + 1,)).copy()
        rwa = np.ctypeslib.as_array(rw, shape=(max(nnz.value, 1),))[: nnz.value].copy()
        return n.value, nnz.value, cpa, rwa

    def build_bvss(self, full_padding: bool) -> None:
        _rcheck(rlib().ref_bvss_build(self.h, int(full_padding)))

    def bvss(self) -> dict:
        n, R, V = C.c_uint32(), C.c_uint32(), C.c_uint32()
        S = C.c_uint64()
        div = C.c_double()
        ssp, v2r, rp, ri, mk = P64(), P32(), P32(), P32(), P32()
        _rcheck(rlib().ref_bvss_get(self.h, C.byref(n), C.byref(R), C.byref(V), C.byref(S), C.byref(div),
                                    C.byref(ssp), C.byref(v2r), C.byref(rp), C.byref(ri), C.byref(mk)))

        def arr(p, k):
            return np.ctypeslib.as_array(p, shape=(max(k, 1),))[:k].copy()

        return {"n": n.value, "update_divergence": div.value,
                "slice_set_ptrs": arr(ssp, V.value + 1), "virtual_to_real": arr(v2r, V.value),
                "real_ptrs": arr(rp, R.value + 1), "row_ids": arr(ri, S.value), "masks": arr(mk, S.value // 4)}

    def bvss_sizes(self) -> tuple[int, int, int, int]:
        """(n, real slice sets R, virtual slice sets V, slices S) of the
        built BVSS (no array copies)."""
        n, R, V = C.c_uint32(), C.c_uint32(), C.c_uint32()
        S = C.c_uint64()
        div = C.c_double()
        ssp, v2r, rp, ri, mk = P64(), P32(), P32(), P32(), P32()
        _rcheck(rlib().ref_bvss_get(self.h, C.byref(n), C.byref(R), C.byref(V), C.byref(S), C.byref(div),
                                    C.byref(ssp), C.byref(v2r), C.byref(rp), C.byref(ri), C.byref(mk)))
        return n.value, R.value, V.value, S.value

    def bvss_slices(self) -> int:
        """Slice count of the built BVSS (no array copies)."""
        return self.bvss_sizes()[3]

    def upload_bytes(self, kind: str, nnz: int) -> int:
        """Bytes the reference's stock hostCode copies host -> device on every
        call: the BVSS arrays (slice-set pointers 8 B, virtual-to-real 4 B
        per vset, real pointers, 4-byte row ids, one mask word per 4
        slices), plus for BFS the pull CSR (BFS/BVSSBFSKernel.cuh:1394-1401)
        and for CC the initial labels and vset queue
        (CC/BVSSCCKernel.cuh:1154-1203)."""
        n, R, V, S = self.bvss_sizes()
        b = 8 * (V + 1) + 4 * V + 4 * (R + 1) + 4 * S + S
        return b + (4 * (n + 1) + 4 * nnz if kind == "bfs" else 4 * n + 4 * V)

    def bfs_variant(self) -> int:
        v = C.c_int()
        _rcheck(rlib().ref_bfs_variant(self.h, C.byref(v)))
        return v.value

    def bfs(self, src: int, n: int):
        out = np.empty(n, dtype=np.uint32)
        t = C.c_double()
        tl, nv = C.c_uint32(), C.c_uint32()
        _rcheck(rlib().ref_bfs(self.h, src, _p32(out), C.byref(t), C.byref(tl), C.byref(nv)))
        return out, t.value, tl.value, nv.value

    def cc(self, n: int):
        out = np.empty(n, dtype=np.uint32)
        t = C.c_double()
        k = C.c_uint32()
        _rcheck(rlib().ref_cc(self.h, _p32(out), C.byref(t), C.byref(k)))
        return out, t.value, k.value

    def cc_raw(self, n: int):
        out = np.empty(n, dtype=np.uint32)
        t = C.c_double()
        _rcheck(rlib().ref_cc_raw(self.h, _p32(out), C.byref(t)))
        return out, t.value
