"""The N>1 host path of bench.py on CPU with gloo (world size 2): rank 0
builds the graph and writes the caches, rank 1 waits for them and loads
identical arrays; timings are reduced with MAX over ranks, sources are the
same on every replica."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, cache, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    bench.WORKLOADS["tiny"] = ("bfs", ("rmat", 12, 8), "jaccard", 1024, 16, "test")
    csc, bvss, csr, sources = bench.prepare("tiny", Path(cache), rank, world)
    a = bvss.arrays()
    digest = torch.tensor([int(a["row_ids"].astype(np.int64).sum()), int(a["masks"].astype(np.int64).sum()),
                           int(sources.astype(np.int64).sum()), csc.nnz], dtype=torch.int64)
    gathered = [torch.zeros_like(digest) for _ in range(world)]
    dist.all_gather(gathered, digest)
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        np.save(out, np.stack([g.numpy() for g in gathered] + [np.full(4, t.item(), dtype=np.int64)]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_share_the_graph_cache(tmp_path):
    out = str(tmp_path / "res.npy")
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path / "cache"), out), nprocs=2, join=True,
                       start_method="spawn")
    res = np.load(out)
    assert np.array_equal(res[0], res[1])  # both replicas hold identical BVSS and sources
    assert res[0][3] > 0
    assert res[2][0] == 2  # max over ranks
