"""B200-native BLEST: BVSS BFS / CC / multi-source BFS on sm_100a.

Layers:
  - C++ host layer (CSC, RCM / windowed-Jaccard orderings, BVSS builder) and
    hand-written sm_100a kernels, in libblest_b200.so behind the C ABI of
    include/blest.h;
  - blest_b200.graph: Python objects over that ABI;
  - include/blest_kernels.hpp: the reference's plugin interface (BFSKernel /
    CCKernel / MBFSKernel with hostCode / run) over the same ABI, for C++
    drivers;
  - blest_b200.server: continuous-batching query server;
  - blest_b200.autotune: launch-parameter search for BFS and MBFS.
"""
from ._lib import BlestError, lib  # noqa: F401  (raises ImportError if the .so is missing)
from .graph import (Bvss, Csc, Graph, MbfsPlan, Workspace, bfs_params, init, load_ordering, mbfs_batch,  # noqa: F401
                    relabel_dense, save_ordering)

__all__ = ["BlestError", "Bvss", "Csc", "Graph", "MbfsPlan", "Workspace", "bfs_params", "init", "load_ordering",
           "mbfs_batch", "relabel_dense",
           "save_ordering", "lib"]
