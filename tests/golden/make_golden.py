"""Generate the host-layer golden fixtures from the reference itself.

Runs the reference's own CSC classification, orderings (windowed Jaccard,
RCM) and BVSS builder -- compiled from its sources into
oracle/_ref/libblest_ref.so by oracle/Makefile -- on small seeded graphs and
stores inputs and outputs as tests/golden/host_<name>.npz. Needs the
reference sources (run where they are mounted):

    make -C oracle && python tests/golden/make_golden.py

The input graphs come from blest_b200's seeded generators, but every stored
output is the reference's.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle as O  # noqa: E402
from blest_b200 import Csc  # noqa: E402

OUT = Path(__file__).resolve().parent

# name -> (graph factory, ordering, window)
CASES = {
    "rmat10_jaccard": (lambda: Csc.rmat(10, 16, seed=3, permute_seed=5), "jaccard", 256),
    "rmat11_jaccard_w64": (lambda: Csc.rmat(11, 8, seed=11, permute_seed=2), "jaccard", 64),
    "rmat9_natural": (lambda: Csc.rmat(9, 16, seed=4, permute_seed=9), "natural", 0),
    "grid45x37_rcm": (lambda: Csc.grid(45, 37, 0.05, 0.001, seed=2), "rcm", 0),
    "grid40x40_jaccard": (lambda: Csc.grid(40, 40, 0.1, 0.01, seed=6), "jaccard", 128),
    "er1999_rcm": (lambda: Csc.er(1999, 3000, seed=7), "rcm", 0),
    "er2000_natural": (lambda: Csc.er(2000, 2000 * 12, seed=8), "natural", 0),
    "directed_natural": (lambda: _directed(1000, 6000, 12), "natural", 0),
}


def _directed(n: int, m: int, seed: int) -> Csc:
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    keep = src != dst
    pairs = np.unique(np.stack([src[keep], dst[keep]], 1), axis=0)
    return Csc.from_edges(n, pairs[:, 0], pairs[:, 1])


def main() -> None:
    for name, (make, mode, window) in CASES.items():
        g = make()
        n = g.n
        cp, rw = g.col_ptrs.copy(), g.rows.copy()
        ref = O.RefGraph.from_csc(n, cp, rw)
        social = ref.is_social()
        inv = ref.reorder(mode, window=window or 65536)
        full_padding = not social
        ref.build_bvss(full_padding)
        b = ref.bvss()
        _, _, rcp, rrw = ref.csc()
        np.savez_compressed(
            OUT / f"host_{name}.npz",
            n=np.uint32(n), col_ptrs=cp, rows=rw, ordering=np.array(mode), window=np.uint32(window),
            is_social=np.bool_(social), inverse_permutation=inv, reordered_col_ptrs=rcp, reordered_rows=rrw,
            full_padding=np.bool_(full_padding), update_divergence=np.float64(b["update_divergence"]),
            slice_set_ptrs=b["slice_set_ptrs"], virtual_to_real=b["virtual_to_real"], real_ptrs=b["real_ptrs"],
            row_ids=b["row_ids"], masks=b["masks"])
        print(f"{name}: n={n} nnz={rw.size} social={social} V={b['virtual_to_real'].size} S={b['row_ids'].size}")


if __name__ == "__main__":
    main()
