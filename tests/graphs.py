"""Small graph cases shared by the GPU parity tests."""
from __future__ import annotations

import numpy as np

from blest_b200 import Bvss, Csc
from conftest import GOLDEN


def edges_graph(n, edges, undirected=True) -> Csc:
    src, dst = [], []
    for u, v in edges:
        src.append(u)
        dst.append(v)
        if undirected:
            src.append(v)
            dst.append(u)
    return Csc.from_edges(n, src, dst)


def path(n):
    return edges_graph(n, [(i, i + 1) for i in range(n - 1)])


def star(n):
    return edges_graph(n, [(0, i) for i in range(1, n)])


def two_cliques(k):
    e = [(i, j) for i in range(k) for j in range(i + 1, k)]
    e += [(k + i, k + j) for i in range(k) for j in range(i + 1, k)]
    return edges_graph(2 * k + 3, e)  # + 3 isolated vertices


def random_directed(n, m, seed):
    rng = np.random.default_rng(seed)
    s, d = rng.integers(0, n, m), rng.integers(0, n, m)
    keep = s != d
    pairs = np.unique(np.stack([s[keep], d[keep]], 1), axis=0)
    return Csc.from_edges(n, pairs[:, 0], pairs[:, 1])


def prepared(csc: Csc, order: str = "auto", window: int = 65536, full_padding=None):
    """Reorder (as CSC::reorder would), build the BVSS and the pull CSR."""
    csc.reorder(order, window=window)
    b = Bvss.build(csc, full_padding=full_padding)
    return csc, b, csc.transpose()


def golden_prepared(path):
    h = dict(np.load(path))
    n = int(h["n"])
    csc = Csc.from_arrays(n, h["reordered_col_ptrs"], h["reordered_rows"])
    b = Bvss.from_arrays(n, h["slice_set_ptrs"], h["virtual_to_real"], h["real_ptrs"], h["row_ids"], h["masks"],
                         full_padding=bool(h["full_padding"]), update_divergence=float(h["update_divergence"]))
    return csc, b, csc.transpose()


def small_cases():
    """(name, factory) for generated parity cases, including ragged sizes."""
    return [
        ("single_vertex", lambda: prepared(Csc.from_arrays(1, [0, 0], []), "natural")),
        ("two_isolated", lambda: prepared(Csc.from_arrays(2, [0, 0, 0], []), "natural")),
        ("path9", lambda: prepared(path(9), "natural")),
        ("path33_rcm", lambda: prepared(path(33), "rcm")),
        ("path1000_fullpad", lambda: prepared(path(1000), "natural", full_padding=True)),
        ("star257", lambda: prepared(star(257), "natural")),
        ("two_cliques", lambda: prepared(two_cliques(20), "natural")),
        ("directed_300", lambda: prepared(random_directed(300, 1500, 3), "natural")),
        ("rmat14_jaccard", lambda: prepared(Csc.rmat(14, 16, seed=5, permute_seed=2), "jaccard", 4096)),
        ("rmat13_natural_fullpad", lambda: prepared(Csc.rmat(13, 8, seed=6, permute_seed=1), "natural",
                                                    full_padding=True)),
        ("grid101x77_rcm", lambda: prepared(Csc.grid(101, 77, 0.05, 0.001, seed=3), "rcm")),
        ("er5001_natural", lambda: prepared(Csc.er(5001, 40000, seed=4), "natural")),
    ]


def golden_cases():
    return [(p.stem, (lambda p=p: golden_prepared(p))) for p in sorted(GOLDEN.glob("host_*.npz"))]
