#!/usr/bin/env python
"""BLEST B200 benchmark: BFS GTEPS on one B200 (default workload: RMAT scale
24, edge factor 16, Jaccard window 65536, 64 seeded sources).

One "step" = one BFS from each of the workload's sources (64 for RMAT-24).
  value : sum of reached undirected edges / device time of the K timed steps
          (graph resident in HBM, levels written to HBM; CUDA events on the
          launching stream; BVSS is larger than L2, so no flush is needed)
  e2e   : the same metric through the public C-ABI call with HOST buffers:
          each BFS's levels are copied to pinned host memory inside the
          timed region (blest_bfs with BLEST_MEM_HOST)
  --impl reference : the reference's own BVSS kernels (compiled from its
          sources for sm_100a into oracle/_ref) on the identical BVSS,
          timed by its own convention (launch -> cudaDeviceSynchronize)

Multi-GPU (torchrun): replicas -- every rank runs the same workload on its
own GPU (weak scaling); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: (kind, generator, ordering, window, n_sources, description)
    "rmat24": ("bfs", ("rmat", 24, 16), "jaccard", 65536, 64,
               "RMAT scale 24 ef 16 (a,b,c)=(.57,.19,.19) seed 1, symmetrised+dedup, seeded id permutation, "
               "Jaccard window 65536, 64 seeded sources"),
    "rmat16": ("bfs", ("rmat", 16, 16), "jaccard", 65536, 64,
               "RMAT scale 16 ef 16, Jaccard window 65536, 64 seeded sources"),
    "rmat20": ("bfs", ("rmat", 20, 16), "jaccard", 65536, 64, "RMAT scale 20 ef 16, Jaccard window 65536"),
    "rmat22": ("bfs", ("rmat", 22, 16), "jaccard", 65536, 64, "RMAT scale 22 ef 16, Jaccard window 65536"),
    "grid4096": ("bfs", ("grid", 4096, 4096), "rcm", 0, 32,
                 "2D 4096x4096 grid, 5% edges deleted, 0.1% shortcuts, RCM, 32 seeded sources"),
    "er25": ("bfs", ("er", 25, 32), "rcm", 0, 32, "Erdos-Renyi 2^25 vertices avg degree 32, RCM, 32 sources"),
    "cc_rmat24": ("cc", ("rmat", 24, 16), "jaccard", 65536, 0, "connected components, RMAT scale 24"),
    "cc_grid4096": ("cc", ("grid", 4096, 4096), "rcm", 0, 0,
                    "connected components, 2D 4096x4096 grid, 5% edges deleted, 0.1% shortcuts, RCM"),
    "cc_er25": ("cc", ("er", 25, 32), "rcm", 0, 0, "connected components, Erdos-Renyi 2^25 avg degree 32, RCM"),
    "serving": ("serving", None, None, 0, 0,
                "query server: resident graphs RMAT 18/20/22, grid 1024^2, ER 2^22 deg 16; Poisson arrivals, "
                "80% BFS (uniform seeded source) / 20% CC, graph uniform; rate sweep"),
    "mbfs_rmat20": ("mbfs", ("rmat", 20, 16), "jaccard", 65536, 128,
                    "multi-source BFS, RMAT scale 20 ef 16, Jaccard window 65536, 128 seeded sources (one group; "
                    "the profiling case)"),
    "cc_rmat20": ("cc", ("rmat", 20, 16), "jaccard", 65536, 0, "connected components, RMAT scale 20 (profiling case)"),
    "er23": ("bfs", ("er", 23, 32), "rcm", 0, 32,
             "Erdos-Renyi 2^23 vertices avg degree 32, RCM, 32 sources (profiling case of er25)"),
    "grid2048": ("bfs", ("grid", 2048, 2048), "rcm", 0, 32,
                 "2D 2048x2048 grid, 5% edges deleted, 0.1% shortcuts, RCM, 32 sources (profiling case of grid4096)"),
    "mbfs_rmat22": ("mbfs", ("rmat", 22, 16), "jaccard", 65536, 1024,
                    "multi-source BFS, RMAT scale 22 ef 16, Jaccard window 65536, 1024 seeded sources "
                    "in bit-packed groups of 128"),
    "mbfs_multi256": ("mbfs_multi", None, "jaccard", 65536, 8,
                      "256 independent RMAT graphs (a,b,c)=(.57,.19,.19), n = round(2^clip(N(14, 2.43), 10, 18)) "
                      "(RMAT on 2^ceil(log2 n) vertices, seeded permutation, induced on ids < n), edge factor "
                      "uniform 4..32, Jaccard window 65536, 8 seeded sources each; one multi-graph MBFS launch "
                      "replayed from a captured CUDA graph"),
}

SEED = 1


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------- graph prep
def prepare(workload: str, cache_dir: Path, rank: int, world: int):
    """Build (or load from the per-run cache) the reordered CSC, BVSS and
    pull CSR. Rank 0 builds; other ranks wait for the cache files. Workloads
    on the same graph share one cache entry; the sources of every such
    workload's count are sampled when the graph is built."""
    from blest_b200 import Bvss, Csc
    kind, gen, order, window, nsrc, _ = WORKLOADS[workload]
    cache_dir.mkdir(parents=True, exist_ok=True)
    tag = cache_dir / f"{'_'.join(map(str, gen))}_{order}_{window}"
    counts = sorted({w[4] for w in WORKLOADS.values() if w[1:4] == (gen, order, window) and w[4]})
    done = Path(str(tag) + ".ready")
    if rank == 0 and not done.exists():
        t0 = time.time()
        if gen[0] == "rmat":
            csc = Csc.rmat(gen[1], gen[2], 0.57, 0.19, 0.19, seed=SEED, permute_seed=SEED)
        elif gen[0] == "grid":
            csc = Csc.grid(gen[1], gen[2], 0.05, 0.001, seed=SEED)
        else:
            n = 1 << gen[1]
            csc = Csc.er(n, n * gen[2] // 2, seed=SEED)
        t1 = time.time()
        samples = {k: csc.sample_sources(k, SEED) for k in counts}
        inv = csc.reorder(order, window=window or 65536)
        t2 = time.time()
        bvss = Bvss.build(csc)
        t3 = time.time()
        log(f"[prep] {workload}: generate {t1 - t0:.1f}s reorder {t2 - t1:.1f}s bvss {t3 - t2:.1f}s "
            f"n={csc.n} nnz={csc.nnz} social={csc.is_social}")
        csc.save_bin(str(tag) + "_csc.bin")
        bvss.save_bin(str(tag) + "_bvss.bin")
        for k, src in samples.items():
            np.save(str(tag) + f"_sources{k}.npy", inv[src])
        done.write_text("ok")
    else:
        deadline = time.time() + 3600
        while not done.exists():
            if time.time() > deadline:
                raise TimeoutError("graph cache not ready")
            time.sleep(1.0)
        csc = Csc.load_bin(str(tag) + "_csc.bin")
        bvss = Bvss.load_bin(str(tag) + "_bvss.bin")
    sources = np.load(str(tag) + f"_sources{nsrc}.npy") if nsrc else np.zeros(0, np.uint32)
    csr = csc if csc.is_symmetric() else csc.transpose()
    return csc, bvss, csr, sources


def reached_edges(csr_degrees: np.ndarray, levels: np.ndarray) -> int:
    """m_R = 1/2 * sum of degrees of reached vertices (each undirected edge once)."""
    return int(csr_degrees[levels != 0xFFFFFFFF].sum()) // 2


def algorithmic_bytes(bvss_arrays: dict, levels: np.ndarray) -> int:
    """5*S_R + 12*V_R + 4*N_R: slices/vsets of rsets holding a reached vertex,
    plus one 4-byte level per reached vertex."""
    reached = np.nonzero(levels != 0xFFFFFFFF)[0]
    rsets = np.unique(reached >> 3)
    rp = bvss_arrays["real_ptrs"]
    ssp = bvss_arrays["slice_set_ptrs"]
    v_r = int((rp[rsets + 1].astype(np.int64) - rp[rsets]).sum())
    s_r = int((ssp[rp[rsets + 1]].astype(np.int64) - ssp[rp[rsets]].astype(np.int64)).sum())
    return 5 * s_r + 12 * v_r + 4 * reached.size


# ----------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        """Start sampling every 20 ms and wait (up to 3 s) for the first
        reading, so that even a short timed region gets samples; readings
        taken before the region starts are left out of the summary."""
        self.first = 0
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.time() + 3.0
            while not self.lines and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.005)
            self.first = len(self.lines)
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[self.first:] or self.lines[-1:]
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(workload: str):
    """DRAM bytes (read + write) per launch of the workload's dominant kernel
    from one ncu capture, as recorded in profiles/traffic.json (a figure
    scaled from a smaller capture says so in that file); None if absent."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    entry = json.loads(p.read_text()).get(workload)
    return float(entry["bytes_per_launch"]) if entry else None


L2_LARGE = "inputs larger than L2 (BVSS+CSR in HBM), no flush"


def bfs_config(workload, n, nnz, nsrc, edges_per_step, slices, world, l2=L2_LARGE):
    """Workload keys of a BFS line, the same for both arms."""
    return {"workload": workload, "description": WORKLOADS[workload][5], "n": int(n), "nnz_directed": int(nnz),
            "undirected_edges": int(nnz) // 2, "sources_per_step": int(nsrc),
            "reached_edges_per_step": int(edges_per_step), "bvss_slices": int(slices),
            "l2": l2, "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


class L2Flush:
    """Between timed steps, for a graph that fits in L2: writes a buffer of
    twice the L2 size on the timing stream, outside the steps' events, so
    every step starts with the graph out of L2. A no-op for larger graphs."""

    def __init__(self, graph_bytes: int, stream, dev: int):
        import torch
        l2 = int(torch.cuda.get_device_properties(dev).L2_cache_size)
        self.active = graph_bytes < 2 * l2
        self.stream = stream
        self.buf = torch.empty(2 * l2 // 4, dtype=torch.int32, device="cuda") if self.active else None
        self.note = (f"graph {graph_bytes / 1e6:.1f} MB fits in L2 ({l2 / 1e6:.0f} MB): L2 flushed between timed "
                     f"steps (a {2 * l2 / 1e6:.0f} MB write outside the timed events)" if self.active else L2_LARGE)
        self.count = 0

    def __call__(self) -> None:
        if self.active:
            import torch
            self.count += 1
            with torch.cuda.stream(self.stream):
                self.buf.fill_(self.count)


def cc_config(workload, n, nnz, slices, components, world):
    return {"workload": workload, "description": WORKLOADS[workload][5], "n": int(n), "nnz_directed": int(nnz),
            "bvss_slices": int(slices), "components": int(components),
            "l2": "inputs larger than L2 (BVSS in HBM), no flush",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def generate_oracle(gen):
    """The workload's graph from the oracle's generator (byte-identical to
    the library's), as (n, col_ptrs, rows)."""
    import oracle as O
    if gen[0] == "rmat":
        return O.gen_rmat(gen[1], gen[2], 0.57, 0.19, 0.19, SEED, SEED)
    if gen[0] == "grid":
        return O.gen_grid(gen[1], gen[2], 0.05, 0.001, SEED, 0)
    n = 1 << gen[1]
    return O.gen_er(n, n * gen[2] // 2, SEED, 0)


# ----------------------------------------------------------------- arms
def run_mbfs(args, rank, world):
    """Multi-source BFS GTEPS (sum over sources of reached edges / batch
    time), next to the same sources run one BFS launch each."""
    import torch
    import torch.distributed as dist
    import blest_b200
    from blest_b200 import Graph, Workspace
    from blest_b200 import _lib as L
    import ctypes as C

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    blest_b200.init(dev)
    kind, gen, order, window, nsrc, desc = WORKLOADS[args.workload]
    csc, bvss, csr, sources = prepare(args.workload, Path(args.cache), rank, world)
    g = Graph(bvss, csr)
    n = csc.n
    k = len(sources)
    deg = torch.from_numpy(np.diff(csr.col_ptrs.astype(np.int64))).cuda()
    out = torch.empty((k, n), dtype=torch.int32, device="cuda")
    src = np.ascontiguousarray(sources, dtype=np.uint32)
    tuned = None
    if not args.no_autotune_mbfs:
        from blest_b200.autotune import tune_mbfs
        tuned, table = tune_mbfs(g, sources)
        log(f"[autotune] mbfs best {tuned} ({table[0]['seconds'] * 1e6:.2f} us/source; "
            f"worst {table[-1]['seconds'] * 1e6:.2f})")
        p = L.MbfsParams(tuned["group_width"], tuned["blocks_per_sm"], 0, tuned.get("pull_fraction", 0.0))
    else:
        p = L.MbfsParams(args.group_width, 0, 0)
    st = L.MbfsStats()
    barrier = (lambda: dist.barrier()) if world > 1 else (lambda: None)

    def mbfs_once():
        L.call("blest_mbfs", g._h, src.ctypes.data_as(L.P(L.u32)), k, out.data_ptr(), L.MEM_DEVICE,
               C.byref(p), C.byref(st))

    mbfs_once()
    reached = (out != -1)
    mr = int(((reached.to(torch.int64) * deg).sum(1) // 2).sum().item())
    del reached
    parity = None
    if rank == 0 and not args.skip_check:
        # every source's levels against the oracle's OpenMP BFS
        import oracle as O
        bad = 0
        for i in range(k):
            want, _ = O.bfs_omp(n, csc.col_ptrs, csc.rows, csr.col_ptrs, csr.rows, int(sources[i]), 0)
            if not np.array_equal(out[i].cpu().numpy().view(np.uint32), want):
                bad += 1
                log(f"[parity] MBFS source #{i} differs from the oracle")
        parity = {"sources_checked": k, "mismatches": bad, "against": "oracle bfs_omp (oracle/oracle.c), all sources"}
        if bad:
            raise SystemExit(f"MBFS levels differ from the oracle for {bad} of {k} sources")
    for _ in range(args.warmup):
        mbfs_once()
    barrier()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(dev) as clocks:
        for _ in range(args.steps):
            mbfs_once()
            times.append(st.time)
    barrier()
    ms = sum(times) * 1e3
    ms_t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    value = mr * args.steps * world / (ms * 1e-3) / 1e9

    # plain: one single-source BFS launch per source (same kernel family)
    ws = Workspace(g)
    stream = torch.cuda.Stream()
    lv = torch.empty(n, dtype=torch.int32, device="cuda")
    for s_ in sources[:8]:
        ws.bfs_async(int(s_), lv.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s_ in sources:
        ws.bfs_async(int(s_), lv.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    plain_ms = e0.elapsed_time(e1)
    plain = mr / (plain_ms * 1e-3) / 1e9

    # e2e: public call with host output, one group (128 sources) per step
    k_e = min(k, 128)
    host = np.empty((k_e, n), dtype=np.uint32)
    t0 = time.perf_counter()
    e_steps = max(1, args.steps)
    for _ in range(e_steps):
        L.call("blest_mbfs", g._h, src.ctypes.data_as(L.P(L.u32)), k_e, host.ctypes.data, L.MEM_HOST,
               C.byref(p), C.byref(st))
    e_secs = time.perf_counter() - t0
    mr_e = 0
    hdeg = np.diff(csr.col_ptrs.astype(np.int64))
    for i in range(k_e):
        mr_e += int(hdeg[host[i] != 0xFFFFFFFF].sum()) // 2
    e2e = mr_e * e_steps / e_secs / 1e9
    peak, peak_kind = measured_peak()
    out_bytes = 4 * k * n
    achieved = out_bytes / (ms / args.steps * 1e-3) / 1e9
    return {
        "metric": "batched MBFS GTEPS (sum over sources of reached edges / batch time)",
        "value": round(value, 3), "unit": "GTEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator; see config)",
        "config": {"workload": args.workload, "description": desc, "n": n, "sources_per_step": k,
                   "group_width": p.group_width, "blocks_per_sm": p.blocks_per_sm or "max",
                   "pull_fraction": p.pull_fraction or 1 / 64,
                   "autotuned": tuned is not None, "reached_edges_per_step": mr,
                   "plain_one_launch_per_source_gteps": round(plain, 3),
                   "speedup_vs_plain": round(value / world / plain, 2),
                   "output_bytes_per_step": out_bytes,
                   "l2": "inputs and outputs larger than L2, no flush"},
        "e2e": {"value": round(e2e, 3), "unit": "GTEPS", "h2d_bytes_per_step": 4 * k_e,
                "d2h_bytes_per_step": 4 * k_e * n, "note": f"host output, {k_e} sources per step, host wall time"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": profiled_traffic(args.workload),
                     "algorithmic_bytes_per_launch": out_bytes, "note": "output levels only (lower bound)"},
        "clocks": clocks.summary(),
        "parity": parity,
    }


MULTI_GRAPHS = 256
MULTI_SOURCES = 8
MULTI_SIGMA = 4.0 / 1.6449  # log2-space sigma: 5th..95th percentile of N(14, sigma) = 10..18


def multi_graph_specs(count: int = MULTI_GRAPHS):
    """(n, edge factor) of the batch: n = round(2^clip(N(14, sigma), 10, 18)),
    edge factor uniform in 4..32, from the recorded seed."""
    rng = np.random.default_rng(SEED)
    exps = np.clip(rng.normal(14.0, MULTI_SIGMA, count), 10.0, 18.0)
    ns = np.round(2.0 ** exps).astype(np.int64)
    efs = rng.integers(4, 33, count)
    return [(int(n), int(ef)) for n, ef in zip(ns, efs)]


def rmat_n(n: int, ef: int, seed: int):
    """RMAT graph on exactly n vertices: the subgraph induced by ids [0, n)
    of a seeded-permuted RMAT graph of 2^ceil(log2 n) vertices whose edge
    factor is raised by 2^s / n, so that about n * ef edges survive."""
    from blest_b200 import Csc
    s = max(1, int(np.ceil(np.log2(n))))
    ef2 = max(1, int(round(ef * (1 << s) / n)))
    big = Csc.rmat(s, ef2, 0.57, 0.19, 0.19, seed=seed, permute_seed=seed)
    if big.n == n:
        return big
    cp = big.col_ptrs.astype(np.int64)
    rows = big.rows
    col = np.repeat(np.arange(big.n, dtype=np.int64), np.diff(cp))
    keep = (col < n) & (rows < n)
    ncp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(col[keep], minlength=n)[:n], out=ncp[1:])
    return Csc.from_arrays(n, ncp.astype(np.uint32), np.ascontiguousarray(rows[keep], dtype=np.uint32))


def _multi_worker_init():
    os.environ["OMP_NUM_THREADS"] = "2"


def _build_multi_graph(job):
    """One graph of the batch: generate, sample k sources (original ids),
    Jaccard-reorder, save the CSC; returns the sources in reordered ids.
    (Its BVSS is built on the device when the graph is uploaded.)"""
    i, n, ef, k, tag = job
    csc = rmat_n(n, ef, SEED + 1 + i)
    s = csc.sample_sources(k, SEED + i)
    inv = csc.reorder("jaccard", window=65536)
    csc.save_bin(f"{tag}/g{i}_csc.bin")
    return i, np.asarray(inv[s], dtype=np.uint32)


def prepare_multi(cache_dir: Path, rank: int, count: int = MULTI_GRAPHS, k: int = MULTI_SOURCES):
    """The batch's graphs (Jaccard-reordered CSCs) and k sources each, built
    by rank 0 into the cache and loaded by every rank."""
    from blest_b200 import Csc
    tag = cache_dir / f"mbfs_multi{count}_v2"
    done = tag / "ready"
    if rank == 0 and not done.exists():
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        tag.mkdir(parents=True, exist_ok=True)
        t0 = time.time()
        specs = multi_graph_specs(count)
        jobs = [(i, n, ef, k, str(tag)) for i, (n, ef) in sorted(enumerate(specs), key=lambda x: -x[1][0] * x[1][1])]
        workers = max(1, min(16, (os.cpu_count() or 2) // 2))
        # spawn: the parent already holds a CUDA context
        with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn"), initializer=_multi_worker_init) as ex:
            res = dict(ex.map(_build_multi_graph, jobs))
        np.save(str(tag / "sources.npy"), np.stack([res[i] for i in range(count)]).astype(np.uint32))
        done.write_text("ok")
        log(f"[prep] mbfs_multi{count}: {time.time() - t0:.1f}s on {workers} processes")
    else:
        deadline = time.time() + 3600
        while not done.exists():
            if time.time() > deadline:
                raise TimeoutError("graph cache not ready")
            time.sleep(1.0)
    graphs = [Csc.load_bin(str(tag / f"g{i}_csc.bin")) for i in range(count)]
    return graphs, np.load(str(tag / "sources.npy"))


def run_mbfs_multi(args, rank, world):
    """Many graphs in one persistent launch: 256 RMAT graphs of lognormal
    size, 8 sources each, run as one multi-graph MBFS plan replayed from a
    captured CUDA graph; next to the same (graph, source) pairs run one
    single-source BFS launch each, and one MBFS launch per graph."""
    import torch
    import torch.distributed as dist
    import blest_b200
    from blest_b200 import Graph, MbfsPlan, Workspace

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    blest_b200.init(dev)
    kind, gen, order, window, nsrc, desc = WORKLOADS[args.workload]
    t0 = time.time()
    cscs, sources = prepare_multi(Path(args.cache), rank, MULTI_GRAPHS, nsrc)
    t_prep = time.time() - t0
    # the BVSS of every graph is built on the device at upload
    t1 = time.time()
    graphs = [Graph.from_csc(c) for c in cscs]
    t_upload = time.time() - t1
    from blest_b200 import Bvss
    ns = [c.n for c in cscs]
    k = sources.shape[1]
    total = sum(ns) * k
    out = torch.empty(total, dtype=torch.int32, device="cuda")
    views, o = [], 0
    for n in ns:
        views.append(out[o:o + k * n].view(k, n))
        o += k * n
    barrier = (lambda: dist.barrier()) if world > 1 else (lambda: None)

    def make(p):
        return MbfsPlan([(g, sources[i], views[i].data_ptr()) for i, g in enumerate(graphs)], **p)

    # autotune: CTAs per SM and the pull threshold (8 sources fill one
    # 32-wide group)
    table = []
    best = None
    for bps in (1, 2):
        for pf in (1 / 16, 1 / 64, 1 / 256):
            p = {"group_width": 32, "blocks_per_sm": bps, "pull_fraction": pf}
            plan = make(p)
            plan.run()
            t = min(plan.run().time for _ in range(3))
            table.append((t, p))
            if best is None or t < best[0]:
                best = (t, p)
            plan.close()
    tuned = best[1]
    log(f"[autotune] multi-graph plan best {tuned}: {best[0] * 1e3:.3f} ms (worst {max(table, key=lambda r: r[0])[0] * 1e3:.3f})")
    plan = make(tuned)
    info = plan.info()
    plan.run()
    # reached edges and algorithmic bytes per step, from the levels
    mr, s_r, v_r, n_r = 0, 0, 0, 0
    for csc, lv in zip(cscs, views):
        bvss = Bvss.build_device(csc)  # for the algorithmic-byte count only
        deg = torch.from_numpy(np.diff(csc.col_ptrs.astype(np.int64))).cuda()
        reached = lv != -1
        mr += int(((reached.to(torch.int64) * deg).sum(1) // 2).sum().item())
        n_r += int(reached.sum().item())
        anyr = reached.any(0).cpu().numpy()
        rsets = np.unique(np.nonzero(anyr)[0] >> 3)
        a = bvss.arrays()
        rp, ssp = a["real_ptrs"], a["slice_set_ptrs"]
        v_r += int((rp[rsets + 1].astype(np.int64) - rp[rsets]).sum())
        s_r += int((ssp[rp[rsets + 1]].astype(np.int64) - ssp[rp[rsets]].astype(np.int64)).sum())
    algo = 5 * s_r + 12 * v_r + 4 * n_r
    parity = None
    if rank == 0 and not args.skip_check:
        # every (graph, source) pair against the oracle
        import oracle as O
        bad = 0
        host_levels = out.cpu().numpy().view(np.uint32)
        o = 0
        for i, csc in enumerate(cscs):
            lv = host_levels[o:o + k * csc.n].reshape(k, csc.n)
            o += k * csc.n
            for j in range(k):
                want = O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, int(sources[i][j]))
                if not np.array_equal(lv[j], want):
                    bad += 1
                    log(f"[parity] multi-graph MBFS graph {i} source {j} differs from the oracle")
        parity = {"sources_checked": int(k * len(cscs)), "mismatches": bad,
                  "against": "oracle bfs_csc (oracle/oracle.c), every (graph, source) pair"}
        if bad:
            raise SystemExit(f"multi-graph MBFS levels differ from the oracle for {bad} pairs")
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        plan.run()
    barrier()
    torch.cuda.synchronize()
    kern = []
    with ClockSampler(dev) as clocks:
        t_start = time.perf_counter()
        for _ in range(args.steps):
            plan.launch()
            kern.append(plan.sync().time)
        wall = time.perf_counter() - t_start
    barrier()
    ms_t = torch.tensor([sum(kern) * 1e3], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    value = mr * args.steps * world / (ms * 1e-3) / 1e9

    # plain: one single-source BFS launch per (graph, source)
    wss = [Workspace(g) for g in graphs]
    st = torch.cuda.Stream()
    scratch = torch.empty(max(ns), dtype=torch.int32, device="cuda")
    for i in range(min(4, len(graphs))):
        wss[i].bfs_async(int(sources[i][0]), scratch.data_ptr(), st.cuda_stream)
    st.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for i, w in enumerate(wss):
        for j in range(k):
            w.bfs_async(int(sources[i][j]), scratch.data_ptr(), st.cuda_stream)
    e1.record(st)
    st.synchronize()
    plain_ms = e0.elapsed_time(e1)
    plain = mr / (plain_ms * 1e-3) / 1e9
    for w in wss:
        w.close()
    # one MBFS launch per graph (blest_mbfs_ws on each graph in turn)
    from blest_b200 import _lib as L
    import ctypes as C
    pm = L.MbfsParams(32, tuned["blocks_per_sm"], 0, tuned["pull_fraction"])
    stt = L.MbfsStats()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for i, g in enumerate(graphs):
        src = np.ascontiguousarray(sources[i], dtype=np.uint32)
        L.call("blest_mbfs", g._h, src.ctypes.data_as(L.P(L.u32)), k, views[i].data_ptr(), L.MEM_DEVICE,
               C.byref(pm), C.byref(stt))
    per_graph_s = time.perf_counter() - t1
    per_graph = mr / per_graph_s / 1e9

    # e2e: new sources (H2D) each step, replay, all levels to pinned host memory
    pinned = torch.empty(total, dtype=torch.int32, pin_memory=True)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        for i in range(len(graphs)):
            plan.set_sources(i, sources[i])
        plan.launch()
        plan.sync()
        pinned.copy_(out, non_blocking=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = ev0.elapsed_time(ev1)
    e2e = mr * args.steps / (e2e_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    kern_s = float(np.mean(kern))
    achieved = algo / kern_s / 1e9
    plan.close()
    return {
        "metric": "batched MBFS GTEPS, many graphs in one launch (sum over (graph, source) of reached edges / batch time)",
        "value": round(value, 3), "unit": "GTEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator; see config)",
        "config": {"workload": args.workload, "description": desc, "graphs": len(graphs),
                   "sources_per_graph": k, "vertices_total": int(sum(ns)),
                   "n_min": int(min(ns)), "n_median": int(np.median(ns)), "n_max": int(max(ns)),
                   "nnz_total": int(sum(c.nnz for c in cscs)), "joined_n": int(info.n),
                   "captured_cuda_graph": bool(info.captured), "grid_blocks": int(info.grid_blocks),
                   "autotuned": tuned, "autotune_table_ms": [[round(t * 1e3, 3), p] for t, p in table],
                   "reached_edges_per_step": mr,
                   "plain_one_launch_per_source_gteps": round(plain, 3),
                   "speedup_vs_plain": round(value / world / plain, 2),
                   "one_mbfs_launch_per_graph_gteps": round(per_graph, 3),
                   "speedup_vs_per_graph": round(value / world / per_graph, 2),
                   "host_wall_ms_per_step": round(wall * 1e3 / args.steps, 4),
                   "prep_seconds": round(t_prep, 1),
                   "upload_with_device_bvss_seconds": round(t_upload, 2),
                   "l2": "outputs larger than L2, no flush"},
        "e2e": {"value": round(e2e, 3), "unit": "GTEPS", "h2d_bytes_per_step": 4 * int(sources.size),
                "d2h_bytes_per_step": 4 * total},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": profiled_traffic(args.workload),
                     "algorithmic_bytes_per_launch": algo, "avg_launch_ms": round(kern_s * 1e3, 4)},
        "clocks": clocks.summary(),
        "parity": parity,
    }


SERVING_GRAPHS = [
    ("rmat18", ("rmat", 18, 16), "jaccard"), ("rmat20", ("rmat", 20, 16), "jaccard"),
    ("rmat22", ("rmat", 22, 16), "jaccard"), ("grid1024", ("grid", 1024, 1024), "rcm"),
    ("er22", ("er", 22, 16), "rcm"),
]
SERVING_GRAPHS_FULL = SERVING_GRAPHS[:3] + [("rmat24", ("rmat", 24, 16), "jaccard"), SERVING_GRAPHS[3],
                                            ("grid4096", ("grid", 4096, 4096), "rcm"), SERVING_GRAPHS[4],
                                            ("er24", ("er", 24, 32), "rcm")]


SERVING_FULL_DESCRIPTION = ("query server: 8 resident graphs, RMAT scales 18/20/22/24, grids 1024^2 and 4096^2, "
                            "ER 2^22 deg 16 and 2^24 deg 32; Poisson arrivals, 80% BFS (uniform seeded source) / "
                            "20% CC, graph uniform; every result copied to pinned host memory; rate sweep")


def build_graph(gen, order):
    from blest_b200 import Bvss, Csc
    if gen[0] == "rmat":
        csc = Csc.rmat(gen[1], gen[2], 0.57, 0.19, 0.19, seed=SEED, permute_seed=SEED)
    elif gen[0] == "grid":
        csc = Csc.grid(gen[1], gen[2], 0.05, 0.001, seed=SEED)
    else:
        n = 1 << gen[1]
        csc = Csc.er(n, n * gen[2] // 2, seed=SEED)
    csc.reorder(order, window=65536)
    return csc, Bvss.build(csc)


def run_serving(args, rank, world):
    """Open-loop Poisson load on the query server, swept over arrival rates."""
    import threading
    import torch
    import blest_b200
    from blest_b200 import Graph
    from blest_b200.server import Server

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    blest_b200.init(dev)
    specs = SERVING_GRAPHS_FULL if args.serving_full else SERVING_GRAPHS
    graphs = []
    for name, gen, order in specs:
        t0 = time.time()
        csc, bvss = build_graph(gen, order)
        g = Graph(bvss, csc)
        srcs = csc.sample_sources(1024, SEED)
        # reached undirected edges per pool source, from multi-source BFS
        deg = torch.from_numpy(np.diff(csc.col_ptrs.astype(np.int64))).cuda()
        lv = torch.empty((128, csc.n), dtype=torch.int32, device="cuda")
        mr = []
        for i in range(0, len(srcs), 128):
            chunk = np.ascontiguousarray(srcs[i:i + 128], dtype=np.uint32)
            import ctypes as C
            from blest_b200 import _lib as L
            L.call("blest_mbfs", g._h, chunk.ctypes.data_as(L.P(L.u32)), chunk.size, lv.data_ptr(), L.MEM_DEVICE,
                   None, None)
            mr += ((lv[:chunk.size] != -1).to(torch.int64) * deg).sum(1).div(2, rounding_mode="floor").tolist()
        del lv
        graphs.append((name, csc, g, np.array(mr, dtype=np.int64), srcs))
        log(f"[serving] {name}: n={csc.n} nnz={csc.nnz} ({time.time() - t0:.1f}s)")
    # result buffers, recycled once a result has been consumed: pinned host
    # memory (the result crosses PCIe) or device memory (it stays in HBM for
    # a consumer on the GPU)
    def make_pools(device: bool):
        """Result buffers per graph: enough that the client rarely waits for
        one (it waits only when every buffer of a graph holds a request in
        flight), capped per graph at --pool-gb of device memory, or
        --host-pool-gb of pinned host memory (at most a quarter of the
        host's available RAM over all graphs)."""
        if device:
            cap = args.pool_gb * 1e9
        else:
            import psutil
            cap = min(args.host_pool_gb * 1e9, 0.25 * psutil.virtual_memory().available / len(graphs))
        pools = []
        for _, csc, _, _, _ in graphs:
            q = []
            for _ in range(max(8, min(args.buffers, int(cap // (4 * csc.n))))):
                if device:
                    q.append(torch.empty(csc.n, dtype=torch.int32, device="cuda"))
                else:
                    q.append(torch.empty(csc.n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32))
            pools.append(q)
        return pools

    # parity through the server: one BFS and one CC request per graph
    # against the oracle (outside the sweep)
    parity = None
    if not args.skip_check:
        import oracle as O
        srv = Server(lanes=args.lanes, max_batch=128)
        bad = 0
        for name, csc, g, _, srcs in graphs:
            gid = srv.add_graph(g)
            s0 = int(srcs[0])
            tb, tc = srv.submit_bfs(gid, s0), srv.submit_cc(gid)
            if not np.array_equal(tb.result(600), O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, s0)):
                bad += 1
                log(f"[parity] serving BFS on {name} differs from the oracle")
            if not np.array_equal(tc.result(600), O.cc_csc(csc.n, csc.col_ptrs, csc.rows)):
                bad += 1
                log(f"[parity] serving CC on {name} differs from the oracle")
        srv.close()
        parity = {"requests_checked": 2 * len(graphs), "mismatches": bad,
                  "against": "oracle bfs_csc / cc_csc, one BFS and one CC request per graph"}
        if bad:
            raise SystemExit(f"{bad} serving results differ from the oracle")
    rates = [float(r) for r in args.rates.split(",")]
    modes = {"host": [False], "device": [True], "both": [False, True]}[args.serving_results]
    sweeps = {}
    for device_results in modes:
        pools = make_pools(device_results)
        sweeps["device" if device_results else "host"] = serving_sweep(args, graphs, pools, rates, Server)
        if device_results and args.compare_always and not args.always_batch:
            # the same device-result sweep with every pending group batched
            sweeps["device_always"] = serving_sweep(args, graphs, pools, rates, Server, always_batch=True)
        del pools
        torch.cuda.empty_cache()
    # value: results in device memory (the result stays in HBM, as `value`
    # keeps inputs and outputs resident for the other workloads); e2e: every
    # result copied to pinned host memory
    sweep = sweeps.get("device") or sweeps["host"]
    head = sweep[min(1, len(sweep) - 1)]
    host = sweeps.get("host")
    ehead = host[min(1, len(host) - 1)] if host else None
    return {
        "metric": "serving p50 latency (ms, open loop: due time to completion) at the sweep's second rate; p50/p99, "
                  "throughput and GTEPS per rate in config.sweep",
        "value": head["p50_ms"], "unit": "ms", "n_gpus": 1, "steps": len(sweep), "warmup": 0,
        "ms_per_step": None, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded generators; Poisson arrivals from a fixed seed)",
        "config": {"workload": "serving",
                   "description": (SERVING_FULL_DESCRIPTION if args.serving_full else WORKLOADS["serving"][5]),
                   "graphs": [x[0] for x in graphs], "lanes": args.lanes, "max_batch": 128,
                   "batch_policy": "always" if args.always_batch else "adaptive",
                   "sweep": sweep, "sweep_host_results": host,
                   "sweep_always_batch": sweeps.get("device_always"),
                   "result_memory": "sweep: device buffers (results stay in HBM for a consumer on the GPU); "
                                    "sweep_host_results: pinned host buffers (each result crosses PCIe)"},
        "e2e": ({"value": ehead["p50_ms"], "unit": "ms", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                 "note": "the same sweep with every result copied to pinned host memory; p50 at its second rate"}
                if ehead else None),
        "clocks": head.get("clocks"),
        "parity": parity,
    }


def serving_sweep(args, graphs, pools, rates, Server, always_batch=None):
    """Open-loop Poisson arrivals at each rate; returns one record per rate.

    Request i is due at its Poisson arrival time and the client submits it
    then, into a free result buffer of its graph. When every buffer of that
    graph holds a request in flight, the request waits in the graph's
    client-side backlog (arrivals for the other graphs go on) and is
    submitted as soon as a buffer of its graph is recycled. A consumer
    thread takes finished tickets from the server's completion queue in
    completion order and recycles their buffers at once. Latency p50/p99 run
    from the due time to completion (open loop, backlog wait included); the
    server's own figures (from submission) are reported beside them."""
    import collections
    import threading
    rng = np.random.default_rng(SEED)
    sweep = []
    for lam in rates:
        srv = Server(lanes=args.lanes, max_batch=128, completion_queue=True,
                     always_batch=args.always_batch if always_batch is None else always_batch)
        gids = [srv.add_graph(g) for _, _, g, _, _ in graphs]
        nreq = int(min(args.requests, max(50, lam * args.seconds)))
        gaps = rng.exponential(1.0 / lam, nreq)
        kinds = rng.random(nreq) < 0.8
        which = rng.integers(0, len(graphs), nreq)
        pick = rng.integers(0, 1 << 30, nreq)  # source of a BFS request: pick % pool size
        inflight = {}  # ticket id -> (graph index, pool source index, buffer, client delay s)
        backlog = [collections.deque() for _ in graphs]  # (request, due) waiting for a buffer
        free = [list(p) for p in pools]
        lock = threading.Lock()
        lat, edges, failed = [], [0], [0]
        left = [nreq]
        waited = [0, 0.0]  # requests that waited for a buffer, their summed wait

        def submit(i, buf, due):  # with the lock held
            gi = int(which[i])
            si = -1
            if kinds[i]:
                src = graphs[gi][4]
                si = int(pick[i] % len(src))
                t = srv.submit_bfs(gids[gi], int(src[si]), out=buf)
            else:
                t = srv.submit_cc(gids[gi], out=buf)
            inflight[t.id] = (gi, si, buf, time.perf_counter() - due)

        def consume():
            while True:
                with lock:
                    if left[0] == 0:
                        return
                got = srv.next_done(0.05)
                if got is None:
                    continue
                tid, info = got
                with lock:
                    gi, si, buf, delay = inflight.pop(tid)
                    left[0] -= 1
                    if backlog[gi]:
                        j, due_j = backlog[gi].popleft()
                        waited[0] += 1
                        waited[1] += time.perf_counter() - due_j
                        submit(j, buf, due_j)
                    else:
                        free[gi].append(buf)
                srv.release(tid)
                if info.status != 0:
                    failed[0] += 1
                else:
                    lat.append(info.done_s - info.submit_s + delay)
                    if si >= 0:
                        edges[0] += int(graphs[gi][3][si])

        cons = threading.Thread(target=consume)
        cons.start()
        with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
            t_start = time.perf_counter()
            due = t_start
            for i in range(nreq):
                due += gaps[i]
                while time.perf_counter() < due:
                    pass
                gi = int(which[i])
                with lock:
                    if free[gi]:
                        submit(i, free[gi].pop(), due)
                    else:
                        backlog[gi].append((i, due))
            while True:  # the backlog drains through the consumer
                with lock:
                    if left[0] == 0:
                        break
                time.sleep(0.001)
            srv.drain(600)
            wall = time.perf_counter() - t_start
        cons.join()
        st = srv.stats()
        lat_ms = np.sort(np.array(lat)) * 1e3
        pct = lambda q: round(float(lat_ms[min(len(lat_ms) - 1, int(q * (len(lat_ms) - 1) + 0.5))]), 3)
        sweep.append({"rate_per_s": lam, "requests": nreq, "wall_s": round(wall, 3),
                      "throughput_per_s": round(nreq / wall, 1),
                      "p50_ms": pct(0.50), "p99_ms": pct(0.99), "mean_ms": round(float(lat_ms.mean()), 3),
                      "server_p50_ms": round(st["p50_latency_s"] * 1e3, 3),
                      "server_p99_ms": round(st["p99_latency_s"] * 1e3, 3),
                      "waited_for_buffer": waited[0], "buffer_wait_s": round(waited[1], 3),
                      "buffers": [len(p) for p in pools], "jobs": st["jobs"],
                      "batched_requests": st["batched_requests"], "rejected": st["rejected"],
                      "failed": failed[0],
                      "jobs_by_kind": {"bfs": st["jobs_bfs"], "mbfs": st["jobs_mbfs"], "cc": st["jobs_cc"]},
                      "requests_by_kind": {"bfs": st["jobs_bfs"], "mbfs": st["requests_mbfs"],
                                           "cc": st["requests_cc"]},
                      "lane_busy_s": {"bfs": round(st["busy_bfs_s"], 3), "mbfs": round(st["busy_mbfs_s"], 3),
                                      "cc": round(st["busy_cc_s"], 3)},
                      "bfs_gteps": round(edges[0] / wall / 1e9, 3), "clocks": clocks.summary()})
        log(f"[serving] rate {lam}/s: {sweep[-1]}")
        srv.close()
    return sweep


def run_b200(args, rank, world):
    import torch
    import torch.distributed as dist
    import blest_b200
    from blest_b200 import Graph, Workspace, bfs_params
    from blest_b200._lib import MEM_HOST

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    blest_b200.init(dev)
    kind, gen, order, window, nsrc, desc = WORKLOADS[args.workload]
    csc, bvss, csr, sources = prepare(args.workload, Path(args.cache), rank, world)
    g = Graph(bvss, csr)
    info = g.info()
    n = csc.n
    deg = np.diff(csr.col_ptrs.astype(np.int64))
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    ws = Workspace(g)
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    barrier = (lambda: dist.barrier()) if world > 1 else (lambda: None)

    params = bfs_params(args.direction, args.slice_test)
    tuned = None
    if args.autotune:
        from blest_b200.autotune import tune_bfs
        params, table = tune_bfs(g, sources)
        tuned = table[0]["params"]
        log(f"[autotune] best {tuned}: {table[0]['seconds'] * 1e3:.3f} ms/BFS "
            f"(worst {table[-1]['seconds'] * 1e3:.3f})")
    # Outside timing: every source once -- reached edges and algorithmic
    # bytes from its levels, and (rank 0) parity of the levels with the
    # oracle's OpenMP BFS on the host cores, whose run times are also the
    # CPU baseline.
    host_lv = np.empty(n, dtype=np.uint32)
    mr, algo = [], []
    arrays = bvss.arrays()
    check = rank == 0 and not args.skip_check
    parity = {"sources_checked": 0, "mismatches": 0, "against": "oracle bfs_omp (oracle/oracle.c), all sources"}
    cpu_secs, cpu_edges, cpu_used = 0.0, 0, 0
    if check:
        import oracle as O
    for s in sources:
        ws.bfs(int(s), host_lv, sptr, params=params)
        mr.append(reached_edges(deg, host_lv))
        algo.append(algorithmic_bytes(arrays, host_lv))
        if check:
            t = time.perf_counter()
            want, cpu_used = O.bfs_omp(n, csc.col_ptrs, csc.rows, csr.col_ptrs, csr.rows, int(s), 0)
            cpu_secs += time.perf_counter() - t
            cpu_edges += mr[-1]
            parity["sources_checked"] += 1
            if not np.array_equal(host_lv, want):
                parity["mismatches"] += 1
                log(f"[parity] source {int(s)}: {int((host_lv != want).sum())} levels differ from the oracle")
    if parity["mismatches"]:
        raise SystemExit(f"BFS levels differ from the oracle for {parity['mismatches']} of {len(sources)} sources")
    edges_per_step = sum(mr)

    def step(events=None):
        for i, s in enumerate(sources):
            if events is not None:
                events[i][0].record(stream)
            ws.bfs_async(int(s), out.data_ptr(), sptr, params=params)
            if events is not None:
                events[i][1].record(stream)

    def settle(count):
        # settle the oldest `count` calls (every call's record is checked)
        for _ in range(count):
            ws.sync_one()

    flush = L2Flush(int(info.device_bytes_graph), stream, dev)
    for _ in range(args.warmup):
        step()
        settle(len(sources))
    stream.synchronize()
    per_bfs = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in sources] for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    flush()
    with ClockSampler(dev) as clocks:
        t0.record(stream)
        for k in range(args.steps):
            step(per_bfs[k])
            if k + 1 < args.steps:
                flush()
            if k:
                settle(len(sources))  # step k - 1 (step k keeps the GPU busy)
        t1.record(stream)
        stream.synchronize()
    ws.sync()
    barrier()
    torch.cuda.synchronize()
    # with flushes, the timed region is the steps alone (first BFS start to
    # last BFS end of each step)
    ms = (sum(evs[0][0].elapsed_time(evs[-1][1]) for evs in per_bfs) if flush.active else t0.elapsed_time(t1))
    bfs_ms = [e[0].elapsed_time(e[1]) for evs in per_bfs for e in evs]
    ms_t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    value = edges_per_step * args.steps * world / (ms * 1e-3) / 1e9

    # The same BFS calls timed by the reference's convention (host wall
    # clock from launch to synchronisation, one BFS at a time;
    # BFS/BVSSBFSKernel.cuh:1469,1545-1548).
    wall = 0.0
    for _ in range(args.steps):
        for s in sources:
            t = time.perf_counter()
            ws.bfs_async(int(s), out.data_ptr(), sptr, params=params)
            ws.sync()
            wall += time.perf_counter() - t
    wall_t = torch.tensor([wall], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(wall_t, op=dist.ReduceOp.MAX)
    value_wall = edges_per_step * args.steps * world / float(wall_t.item()) / 1e9

    # e2e: the public call with pinned HOST output, copies inside the timed
    # region; the pipelined mode overlaps the copy of BFS i with the kernel
    # of BFS i + 1 (two host buffers, call i settled after call i + 1 is
    # issued).
    bufs = [torch.empty(n, dtype=torch.int32, pin_memory=True) for _ in range(2)]
    bptr = [b.data_ptr() for b in bufs]
    for i, s in enumerate(sources[: min(4, len(sources))]):
        ws.bfs_async(int(s), bptr[i % 2], sptr, out_mem=MEM_HOST, params=params)
        ws.sync()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    j = 0
    for _ in range(args.steps):
        for s in sources:
            ws.bfs_async(int(s), bptr[j % 2], sptr, out_mem=MEM_HOST, params=params)
            if j:
                ws.sync_one()
            j += 1
    ws.sync_one()
    e1.record(stream)
    stream.synchronize()
    e2e_ms_t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_ms_t, op=dist.ReduceOp.MAX)
    e2e_ms = float(e2e_ms_t.item())
    e2e = edges_per_step * args.steps * world / (e2e_ms * 1e-3) / 1e9
    # the copy bound of e2e: one level array per BFS at the measured
    # device-to-host bandwidth into pinned memory
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    bufs[0].copy_(out, non_blocking=True)
    c0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(16):
            bufs[0].copy_(out, non_blocking=True)
    c1.record(stream)
    stream.synchronize()
    d2h_gbs = 16 * 4.0 * n / (c0.elapsed_time(c1) * 1e-3) / 1e9
    copy_bound = edges_per_step / (len(sources) * 4.0 * n / (d2h_gbs * 1e9)) / 1e9
    if check:
        # the last pipelined result must still equal the oracle's
        last = sources[-1]
        want, _ = O.bfs_omp(n, csc.col_ptrs, csc.rows, csr.col_ptrs, csr.rows, int(last), 0)
        if not np.array_equal(bufs[(j - 1) % 2].numpy().view(np.uint32), want):
            raise SystemExit("pipelined host-output BFS differs from the oracle")

    if args.trace_levels and rank == 0:
        # per-level records of a few traced BFS runs (diagnostics, stderr)
        from blest_b200 import _lib as L
        import ctypes as C
        tp = bfs_params(args.direction, args.slice_test, trace=True)
        recs = (L.LevelTrace * 4096)()
        for s in sources[: args.trace_levels]:
            ws.bfs_async(int(s), out.data_ptr(), sptr, params=tp)
            st = ws.sync()
            cnt = L.u32()
            L.call("blest_workspace_trace", ws._h, recs, 4096, C.byref(cnt))
            log(f"[trace] source {int(s)}: {cnt.value - 1} levels, {st.time * 1e3:.3f} ms "
                f"(push {st.push_levels}, pull {st.pull_levels})")
            for i in range(cnt.value - 1):
                r, nx = recs[i], recs[i + 1]
                sweep = f" (sweep {(nx.start_ns - r.sweep_ns) / 1e3:.1f} us)" if r.sweep_ns else ""
                log(f"[trace]   L{r.level:<4d} {'push' if r.direction == 1 else 'pull'} frontier {r.frontier:>9d} "
                    f"units {r.work_units:>10d} {(nx.start_ns - r.start_ns) / 1e3:9.1f} us{sweep}")
    peak, peak_kind = measured_peak()
    avg_bytes = float(np.mean(algo))
    avg_launch_s = float(np.mean(bfs_ms)) * 1e-3
    achieved = avg_bytes / avg_launch_s / 1e9
    traffic = profiled_traffic(args.workload)
    result = {
        "metric": "BFS GTEPS (single-source, direction-optimising BVSS BFS)",
        "value": round(value, 3), "unit": "GTEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator; see config)",
        "config": bfs_config(args.workload, n, csc.nnz, len(sources), edges_per_step, info.no_slices, world,
                             flush.note),
        "impl_detail": {"bfs_params": tuned or f"defaults (alpha 14, beta 24, occupancy grid, "
                                                 f"{args.slice_test} slice test, direction {args.direction})",
                        "device_tiles": int(info.device_tiles),
                        "graph_bytes_hbm": int(info.device_bytes_graph)},
        "value_reference_timing": {"value": round(value_wall, 3), "unit": "GTEPS",
                                   "note": "host wall time launch -> synchronise per BFS, the reference's "
                                           "convention (BFS/BVSSBFSKernel.cuh:1469,1545-1548)"},
        "e2e": {"value": round(e2e, 3), "unit": "GTEPS", "h2d_bytes_per_step": 4 * int(len(sources)),
                "d2h_bytes_per_step": 4 * n * int(len(sources)),
                "note": "blest_bfs_ws with pinned host output, copy of BFS i overlapped with BFS i + 1",
                "d2h_gbs_measured": round(d2h_gbs, 2), "copy_bound_gteps": round(copy_bound, 3),
                "frac_of_copy_bound": round(e2e / world / copy_bound, 3)},
        "gpu_launches": int(len(sources)) * args.steps,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_launch": int(avg_bytes),
                     "avg_launch_ms": round(avg_launch_s * 1e3, 4)},
    }
    if check:
        result["parity"] = parity
    result["clocks"] = clocks.summary()
    if check and not args.no_cpu_baseline:
        result["cpu_baseline"] = {"value": round(cpu_edges / cpu_secs / 1e9, 4), "unit": "GTEPS", "cores": cpu_used,
                                  "kind": "port", "sample": f"{len(sources)} of {len(sources)} sources "
                                                            f"(the parity runs), {cpu_secs:.1f} s"}
    return result


def run_cc(args, rank, world):
    """Connected components by BVSS label propagation: ms per full CC run
    (labels = minimum vertex id of the component), device output; e2e adds
    the labels' device->host copy into pinned memory."""
    import torch
    import torch.distributed as dist
    import blest_b200
    from blest_b200 import Graph, Workspace
    from blest_b200._lib import MEM_HOST

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    blest_b200.init(dev)
    kind, gen, order, window, nsrc, desc = WORKLOADS[args.workload]
    csc, bvss, csr, _ = prepare(args.workload, Path(args.cache), rank, world)
    g = Graph(bvss, csr)
    info = g.info()
    n = csc.n
    barrier = (lambda: dist.barrier()) if world > 1 else (lambda: None)
    ws = Workspace(g)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    lab, st0 = g.cc()
    parity = None
    if rank == 0 and not args.skip_check:
        import oracle as O
        bad = int((lab != O.cc_csc(n, csc.col_ptrs, csc.rows)).sum())
        parity = {"runs_checked": 1, "mismatches": int(bad > 0), "labels_differing": bad,
                  "against": "oracle cc_csc (union-find fixpoint: minimum vertex id per component)"}
        if bad:
            raise SystemExit(f"CC labels differ from the oracle at {bad} vertices")
    for _ in range(args.warmup):
        ws.cc(out.data_ptr(), sptr)
    kern = []
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clocks:
        t0.record(stream)
        for _ in range(args.steps):
            kern.append(ws.cc(out.data_ptr(), sptr).time)
        t1.record(stream)
        stream.synchronize()
    barrier()
    ms_t = torch.tensor([t0.elapsed_time(t1) / args.steps], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())

    pinned = torch.empty(n, dtype=torch.int32, pin_memory=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ws.cc(pinned.data_ptr(), sptr, MEM_HOST)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        ws.cc(pinned.data_ptr(), sptr, MEM_HOST)
    e1.record(stream)
    stream.synchronize()
    e2e_t = torch.tensor([e0.elapsed_time(e1) / args.steps], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)

    # One full pass over the BVSS tiles (5 bytes per slice) plus a label read
    # and write per vertex: the least traffic of any label propagation.
    algo = 5 * int(info.no_slices) + 8 * n
    kern_s = float(np.mean(kern))
    peak, peak_kind = measured_peak()
    achieved = algo / kern_s / 1e9
    result = {
        "metric": "CC time (BVSS label propagation, labels = component minimum id)",
        "value": round(ms, 4), "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator; see config)",
        "config": cc_config(args.workload, n, csc.nnz, info.no_slices, st0.no_components, world),
        "impl_detail": {"iterations": int(st0.iterations)},
        "e2e": {"value": round(float(e2e_t.item()), 4), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 4 * n},
        "gpu_launches": 4 * args.steps,  # init, queue seed, persistent propagation, component count
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": profiled_traffic(args.workload),
                     "algorithmic_bytes_per_launch": algo, "avg_launch_ms": round(kern_s * 1e3, 4)},
        "clocks": clocks.summary(),
        "parity": parity,
    }
    if parity:
        result["parity"] = parity
    if rank == 0 and not args.no_cpu_baseline:
        # the oracle's OpenMP CC on all host cores, the whole graph once
        import oracle as O
        t = time.perf_counter()
        _, used = O.cc_omp(n, csc.col_ptrs, csc.rows)
        secs = time.perf_counter() - t
        result["cpu_baseline"] = {"value": round(secs * 1e3, 2), "unit": "ms", "cores": int(used), "kind": "port",
                                  "sample": f"the whole graph once, {secs:.1f} s"}
    return result


def prepare_reference(workload: str, cache_dir: Path):
    """The workload's graph built by the REFERENCE's own host code through
    oracle/_ref (never libblest_b200.so): the oracle generator's CSC (the
    same bytes as the library's generator), the reference's CSC object and
    classification, its ordering (Jaccard window or RCM), its BVSS builder
    with FULL_PADDING = !social (Benchmark.cuh:113-114, 187-194), and the
    seeded sources mapped to the new ids as Benchmark.cuh:80 does. Like the
    reference's own driver, the reordered CSC is cached with its
    CSC::saveToBinary (and read back with CSC::constructFromBinary), so the
    BFS and CC workloads of one graph reorder it once."""
    import oracle as O
    kind, gen, order, window, nsrc, _ = WORKLOADS[workload]
    cache_dir.mkdir(parents=True, exist_ok=True)
    tag = cache_dir / f"reference_{'_'.join(map(str, gen))}_{order}_{window}"
    counts = sorted({w[4] for w in WORKLOADS.values() if w[1:4] == (gen, order, window) and w[4]})
    t0 = time.time()
    meta = Path(str(tag) + ".json")
    if meta.exists():
        info = json.loads(meta.read_text())
        ref = O.RefGraph.load_csc(str(tag) + "_csc.bin")
        social = bool(info["social"])
        src = np.load(str(tag) + f"_sources{nsrc}.npy") if nsrc else np.zeros(0, np.uint32)
        t1 = t2 = time.time()
    else:
        n, cp, rw = generate_oracle(gen)
        samples = {k: O.sample_sources(n, cp, k, SEED) for k in counts}
        t1 = time.time()
        ref = O.RefGraph.from_csc(n, cp, rw)
        del cp, rw
        social = ref.is_social()
        inv = ref.reorder(order, window or 65536)
        t2 = time.time()
        ref.save_csc(str(tag) + "_csc.bin")
        for k, sk in samples.items():
            np.save(str(tag) + f"_sources{k}.npy", inv[sk].astype(np.uint32))
        meta.write_text(json.dumps({"social": social}))
        src = inv[samples[nsrc]] if nsrc else np.zeros(0, np.uint32)
    ref.build_bvss(full_padding=not social)
    t3 = time.time()
    n, nnz, rcp, rrw = ref.csc()
    slices = int(ref.bvss_slices())
    log(f"[prep:reference] {workload}: generate {t1 - t0:.1f}s reorder {t2 - t1:.1f}s bvss {t3 - t2:.1f}s "
        f"n={n} nnz={nnz} social={social} slices={slices}")
    return ref, n, nnz, rcp, rrw, np.asarray(src, dtype=np.uint32), slices


def run_reference(args, rank, world):
    """The reference's own stock path, independent of this library: its
    host code builds the graph (prepare_reference) and
    BVSSBFSKernel::hostCode / BVSSCCKernel::hostCode (its kernels compiled
    from its sources for sm_100a, oracle/_ref) run it, each call uploading
    the graph and downloading the result as the reference does
    (BFS/BVSSBFSKernel.cuh:1385-1447, 1550). `value` is the reference's own
    timing (launch -> cudaDeviceSynchronize); `e2e` is the wall time of the
    whole hostCode call. Each timed step is a bounded sample of the
    workload's sources (rotating, so all of them are covered); rank 0 only."""
    if rank != 0:
        return None
    import oracle as O
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libblest_ref.so was not built (no reference sources)"}
    kind, gen, order, window, nsrc, desc = WORKLOADS[args.workload]
    if kind in ("mbfs", "mbfs_multi", "serving"):
        return {"impl": "reference", "unavailable": "the reference has no multi-source BFS or serving implementation "
                                                    "(MBFS/BVSSMBFSKernel.cuh is empty; no server)"}
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    ref, n, nnz, cp, rw, sources, slices = prepare_reference(args.workload, Path(args.cache))
    deg = np.diff(cp.astype(np.int64))
    variant = ["BVSSBFS8EnhancedSliceSize8NoMasks4", "FullPad", "LazySwitching", "LazyFullPad"][ref.bfs_variant()]
    if kind == "cc":
        t = time.perf_counter()
        comp, secs0, k0 = ref.cc(n)
        wall0 = time.perf_counter() - t
        parity = None
        if not args.skip_check:
            # the reference's host relabel scrambles labels (CC/BVSSCCKernel.cuh:1282-1287): compare the
            # component count with the oracle's
            want = O.cc_csc(n, cp, rw)
            k_want = int(np.unique(want).size)
            parity = {"runs_checked": 1, "mismatches": int(k0 != k_want), "components": int(k0),
                      "against": "oracle cc_csc component count (the reference's relabelled labels are not a "
                                 "partition, CC/BVSSCCKernel.cuh:1282-1287)"}
        for _ in range(args.warmup - 1):
            ref.cc(n)
        ts, walls = [], []
        with ClockSampler(dev) as clocks:
            for _ in range(args.steps):
                t = time.perf_counter()
                ts.append(ref.cc(n)[1])
                walls.append(time.perf_counter() - t)
        ms = float(np.mean(ts)) * 1e3
        res = {
            "impl": "reference", "metric": "CC time (BVSS label propagation, labels = component minimum id)",
            "value": round(ms, 4), "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32", "data": "synthetic (seeded generator; see config)",
            "config": cc_config(args.workload, n, nnz, slices, k0, 1),
            "impl_detail": {"reference_kernel": "BVSSCC8EnhancedSliceSize8NoMasks4" +
                            ("LazyFullPad" if variant.endswith("FullPad") else "Lazy"),
                            "timing": "BVSSCCKernel::hostCode's own time (launch -> cudaDeviceSynchronize)"},
            "e2e": {"value": round(float(np.mean(walls)) * 1e3, 4), "unit": "ms",
                    "h2d_bytes_per_step": ref.upload_bytes("cc", nnz), "d2h_bytes_per_step": 4 * n,
                    "note": "wall time of the whole stock hostCode call: per-call graph upload, run, label download, "
                            "host relabel"},
            "clocks": clocks.summary(),
        }
        if parity:
            res["parity"] = parity
        if not args.no_cpu_baseline:
            t = time.perf_counter()
            _, used = O.cc_omp(n, cp, rw)
            secs = time.perf_counter() - t
            res["cpu_baseline"] = {"value": round(secs * 1e3, 2), "unit": "ms", "cores": int(used), "kind": "port",
                                   "sample": f"the oracle's OpenMP CC, the whole graph once, {secs:.1f} s (the "
                                             f"reference has no CPU path)"}
        return res

    # Every source once: reached edges, parity against the oracle (the
    # oracle's OpenMP BFS on the host cores, whose times are the CPU
    # baseline), and the first warm-up step.
    mr = {}
    parity = {"sources_checked": 0, "mismatches": 0, "against": "oracle bfs_omp (oracle/oracle.c), all sources"}
    cpu_secs, cpu_edges, cpu_used = 0.0, 0, 0
    for s in sources:
        lv, _, _, _ = ref.bfs(int(s), n)
        mr[int(s)] = reached_edges(deg, lv)
        if not args.skip_check:
            t = time.perf_counter()
            want, cpu_used = O.bfs_omp(n, cp, rw, cp, rw, int(s), 0)
            cpu_secs += time.perf_counter() - t
            cpu_edges += mr[int(s)]
            parity["sources_checked"] += 1
            parity["mismatches"] += int(not np.array_equal(lv, want))
    per_step = max(1, min(args.ref_sources, len(sources)))
    for _ in range(args.warmup - 1):
        ref.bfs(int(sources[0]), n)
    tot_t, tot_wall, tot_e, k = 0.0, 0.0, 0, 0
    with ClockSampler(dev) as clocks:
        for _ in range(args.steps):
            for _ in range(per_step):
                s = int(sources[k % len(sources)])
                k += 1
                t = time.perf_counter()
                _, secs, _, _ = ref.bfs(s, n)
                tot_wall += time.perf_counter() - t
                tot_t += secs
                tot_e += mr[s]
    value = tot_e / tot_t / 1e9
    res = {
        "impl": "reference", "metric": "BFS GTEPS (single-source, direction-optimising BVSS BFS)",
        "value": round(value, 3), "unit": "GTEPS", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(tot_t * 1e3 / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator; see config)",
        "config": bfs_config(args.workload, n, nnz, len(sources), sum(mr.values()), slices, 1,
                             L2_LARGE if 5 * slices + 4 * nnz > 252e6 else
                             "each stock hostCode call uploads the graph first (BFS/BVSSBFSKernel.cuh:1385-1447), "
                             "which leaves it in L2; no flush"),
        "impl_detail": {"reference_kernel": variant,
                        "timing": "BVSSBFSKernel::hostCode's own time: omp_get_wtime launch -> cudaDeviceSynchronize "
                                  "(BFS/BVSSBFSKernel.cuh:1469,1545-1548)"},
        "sample": f"{per_step} of the {len(sources)} sources per timed step, rotating ({k} BFS calls); every source "
                  f"ran once before timing",
        "e2e": {"value": round(tot_e / tot_wall / 1e9, 4), "unit": "GTEPS",
                "h2d_bytes_per_step": ref.upload_bytes("bfs", nnz) * per_step, "d2h_bytes_per_step": 4 * n * per_step,
                "note": "wall time of the whole stock hostCode call: per-call graph upload "
                        "(BFS/BVSSBFSKernel.cuh:1385-1447), run, level download (:1550)"},
        "clocks": clocks.summary(),
    }
    if not args.skip_check:
        res["parity"] = parity
        if not args.no_cpu_baseline:
            res["cpu_baseline"] = {"value": round(cpu_edges / cpu_secs / 1e9, 4), "unit": "GTEPS",
                                   "cores": cpu_used, "kind": "port",
                                   "sample": f"the oracle's OpenMP BFS on all {len(sources)} sources, "
                                             f"{cpu_secs:.1f} s (the reference has no CPU BFS)"}
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="rmat24")
    ap.add_argument("--cache", default="/tmp/blest_bench_cache")
    ap.add_argument("--ref-sources", type=int, default=8,
                    help="reference arm: sources per timed step (each call re-uploads the graph)")
    ap.add_argument("--direction", choices=["auto", "push", "pull"], default="auto",
                    help="BFS direction policy (push-only is the reference's eager kernel's schedule)")
    ap.add_argument("--slice-test", choices=["cuda_core", "mma"], default="cuda_core",
                    help="BFS slice test: CUDA-core byte AND, or the b1 mma.sync m8n8k128 AND+POPC")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-check", action="store_true")
    ap.add_argument("--group-width", type=int, default=128)
    ap.add_argument("--rates", default="100,1000,10000,50000")
    ap.add_argument("--requests", type=int, default=3000)
    ap.add_argument("--seconds", type=float, default=2.0)
    ap.add_argument("--lanes", type=int, default=4)
    ap.add_argument("--serving-full", action="store_true")
    ap.add_argument("--buffers", type=int, default=512,
                    help="serving: most result buffers per graph")
    ap.add_argument("--pool-gb", type=float, default=8.0,
                    help="serving: most GB of device result buffers per graph")
    ap.add_argument("--always-batch", action="store_true",
                    help="serving: coalesce every group of pending BFS requests (no adaptive policy)")
    ap.add_argument("--compare-always", action="store_true",
                    help="serving: also run the device-result sweep with --always-batch, for comparison")
    ap.add_argument("--host-pool-gb", type=float, default=3.0,
                    help="serving: most GB of pinned host result buffers per graph")
    ap.add_argument("--serving-results", choices=["host", "device", "both"], default="both",
                    help="serving: result buffers in pinned host memory, device memory, or a sweep of each")
    ap.add_argument("--autotune", action="store_true", help="tune BFS launch parameters before timing")
    ap.add_argument("--trace-levels", type=int, default=0,
                    help="BFS: log per-level timings of this many traced runs to stderr")
    ap.add_argument("--no-autotune-mbfs", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warmup raised to 3 (minimum)")
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            res = run_reference(args, rank, world)
        elif WORKLOADS[args.workload][0] == "mbfs":
            res = run_mbfs(args, rank, world)
        elif WORKLOADS[args.workload][0] == "mbfs_multi":
            res = run_mbfs_multi(args, rank, world)
        elif WORKLOADS[args.workload][0] == "cc":
            res = run_cc(args, rank, world)
        elif WORKLOADS[args.workload][0] == "serving":
            res = run_serving(args, rank, world) if rank == 0 else None
        else:
            res = run_b200(args, rank, world)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
