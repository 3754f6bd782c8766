"""Autotuner for the BFS / multi-source BFS launch parameters.

Times candidate configurations on a sample of sources with CUDA events and
keeps the fastest: CTAs per SM, the direction-switch thresholds (alpha,
beta) and the slice test (CUDA-core vs b1 MMA) for single-source BFS; the
group width (32/64/128 sources per pass) and CTAs per SM for multi-source
BFS. Levels do not depend on any of these parameters, so the choice is
purely a speed one. Results can be cached in a JSON file keyed by the
graph's shape (n, nnz, slices).
"""
from __future__ import annotations

import itertools
import json
import time
from pathlib import Path

import numpy as np

from . import _lib as L
from .graph import Graph, Workspace, bfs_params

BFS_SPACE = {
    "blocks_per_sm": [1, 2],
    "alpha": [4.0, 14.0, 50.0],
    "beta": [8.0, 24.0, 96.0],
    "slice_test": ["cuda_core", "mma"],
}
MBFS_SPACE = {"group_width": [32, 64, 128], "blocks_per_sm": [1, 2], "pull_fraction": [1 / 256, 1 / 64, 1 / 16]}


def _key(graph: Graph) -> str:
    i = graph.info()
    return f"n{i.n}_nnz{i.nnz}_s{i.no_slices}"


def _load(cache: str | None, key: str, kind: str):
    if not cache or not Path(cache).exists():
        return None
    return json.loads(Path(cache).read_text()).get(kind, {}).get(key)


def _store(cache: str | None, key: str, kind: str, value: dict) -> None:
    if not cache:
        return
    p = Path(cache)
    data = json.loads(p.read_text()) if p.exists() else {}
    data.setdefault(kind, {})[key] = value
    p.write_text(json.dumps(data, indent=1))


def time_bfs(graph: Graph, sources, params: L.BfsParams, repeats: int = 2) -> float:
    """Mean device seconds per BFS (levels to device memory, events on the stream)."""
    import torch
    ws = Workspace(graph)
    out = torch.empty(graph.n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    for s in sources[:2]:
        ws.bfs_async(int(s), out.data_ptr(), stream.cuda_stream, params=params)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(repeats):
        for s in sources:
            ws.bfs_async(int(s), out.data_ptr(), stream.cuda_stream, params=params)
    e1.record(stream)
    stream.synchronize()
    ws.close()
    return e0.elapsed_time(e1) * 1e-3 / (repeats * len(sources))


def tune_bfs(graph: Graph, sources, space: dict | None = None, cache: str | None = None,
             max_sources: int = 8) -> tuple[L.BfsParams, list]:
    """Best single-source BFS parameters for `graph`; returns (params, table)."""
    key = _key(graph)
    hit = _load(cache, key, "bfs")
    if hit:
        return bfs_params(**hit["params"]), hit["table"]
    space = space or BFS_SPACE
    src = list(np.asarray(sources)[:max_sources])
    table = []
    names = list(space)
    for combo in itertools.product(*(space[k] for k in names)):
        kw = dict(zip(names, combo))
        t = time_bfs(graph, src, bfs_params(**kw))
        table.append({"params": kw, "seconds": t})
    table.sort(key=lambda r: r["seconds"])
    best = table[0]["params"]
    _store(cache, key, "bfs", {"params": best, "table": table, "when": time.time()})
    return bfs_params(**best), table


def tune_mbfs(graph: Graph, sources, space: dict | None = None, cache: str | None = None,
              max_sources: int = 256) -> tuple[dict, list]:
    """Best multi-source parameters for `graph` on (a sample of at most
    max_sources of) `sources`; returns (params, table). seconds are per
    source."""
    import ctypes as C

    import torch
    key = _key(graph) + f"_k{len(sources)}"
    hit = _load(cache, key, "mbfs")
    if hit:
        return hit["params"], hit["table"]
    space = space or MBFS_SPACE
    src = np.ascontiguousarray(np.asarray(sources)[:max_sources], dtype=np.uint32)
    out = torch.empty((src.size, graph.n), dtype=torch.int32, device="cuda")
    table = []
    for gw, bps, pf in itertools.product(space["group_width"], space["blocks_per_sm"],
                                         space.get("pull_fraction", [0.0])):
        p = L.MbfsParams(gw, bps, 0, pf)
        st = L.MbfsStats()
        call = lambda: L.call("blest_mbfs", graph._h, src.ctypes.data_as(L.P(L.u32)), src.size,  # noqa: E731
                              out.data_ptr(), L.MEM_DEVICE, C.byref(p), C.byref(st))
        call()
        call()
        table.append({"params": {"group_width": gw, "blocks_per_sm": bps, "pull_fraction": pf},
                      "seconds": st.time / src.size})
    del out
    table.sort(key=lambda r: r["seconds"])
    _store(cache, key, "mbfs", {"params": table[0]["params"], "table": table, "when": time.time()})
    return table[0]["params"], table
