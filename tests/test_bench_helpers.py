"""bench.py's own logic on CPU: the 256-graph batch's size distribution,
RMAT graphs on an exact vertex count, the shared graph cache, the clock
sample summary and the algorithmic-byte count used by the roofline line."""
import numpy as np

import bench
from blest_b200 import Bvss, Csc


def test_multi_graph_specs_follow_the_stated_distribution():
    specs = bench.multi_graph_specs()
    ns = np.array([n for n, _ in specs])
    efs = np.array([e for _, e in specs])
    assert len(specs) == bench.MULTI_GRAPHS == 256
    assert ns.min() >= 1 << 10 and ns.max() <= 1 << 18
    lg = np.log2(ns)
    assert 13.0 < np.median(lg) < 15.0
    assert np.percentile(lg, 5) < 11.0 and np.percentile(lg, 95) > 17.0
    assert efs.min() >= 4 and efs.max() <= 32
    assert specs == bench.multi_graph_specs()  # seeded


def test_rmat_on_an_exact_vertex_count():
    for n, ef in [(3000, 8), (1024, 4), (5000, 20)]:
        g = bench.rmat_n(n, ef, seed=3)
        assert g.n == n
        assert g.is_symmetric()
        cp, rows = g.col_ptrs.astype(np.int64), g.rows
        col = np.repeat(np.arange(n), np.diff(cp))
        assert not np.any(col == rows)  # no self loops
        assert rows.max() < n
        # about n * ef undirected edges survive the induced subgraph
        assert 0.5 * n * ef < g.nnz / 2 < 1.5 * n * ef
    a, b = bench.rmat_n(3000, 8, seed=3), bench.rmat_n(3000, 8, seed=3)
    assert np.array_equal(a.rows, b.rows)


def test_workloads_on_one_graph_share_the_cache(tmp_path):
    saved = dict(bench.WORKLOADS)
    try:
        bench.WORKLOADS["tinyA"] = ("bfs", ("rmat", 10, 8), "jaccard", 1024, 8, "t")
        bench.WORKLOADS["tinyB"] = ("cc", ("rmat", 10, 8), "jaccard", 1024, 0, "t")
        bench.WORKLOADS["tinyC"] = ("mbfs", ("rmat", 10, 8), "jaccard", 1024, 16, "t")
        c1, b1, _, s1 = bench.prepare("tinyA", tmp_path, 0, 1)
        entries = sorted(p.name for p in tmp_path.iterdir())
        c2, b2, _, s2 = bench.prepare("tinyB", tmp_path, 0, 1)
        c3, _, _, s3 = bench.prepare("tinyC", tmp_path, 0, 1)
        assert sorted(p.name for p in tmp_path.iterdir()) == entries  # nothing rebuilt
        assert len(s1) == 8 and len(s2) == 0 and len(s3) == 16
        assert np.array_equal(c1.rows, c2.rows) and np.array_equal(c1.rows, c3.rows)
        assert np.array_equal(b1.arrays()["row_ids"], b2.arrays()["row_ids"])
        deg = np.diff(c1.col_ptrs.astype(np.int64))
        assert np.all(deg[s1] > 0) and np.all(deg[s3] > 0)  # sources have edges
    finally:
        bench.WORKLOADS.clear()
        bench.WORKLOADS.update(saved)


def test_clock_summary_counts_only_readings_inside_the_region():
    cs = bench.ClockSampler(0)
    cs.first = 1
    cs.lines = ["0, 1200, 1965, 300, 0x0, Not Active, Not Active, Not Active, Not Active",
                "0, 1965, 1965, 900, 0x4, Not Active, Not Active, Not Active, Active",
                "0, 1950, 1965, 950, 0x4, Not Active, Not Active, Not Active, Active",
                "garbage line"]
    s = cs.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == 1957.5 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    cs.first = 4  # no reading inside the region: the last one stands in (here unparsable)
    assert cs.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
    cs.first, cs.lines = 1, cs.lines[:2]  # only the pre-region reading and one inside
    assert cs.summary()["samples"] == 1


def test_algorithmic_bytes_and_reached_edges():
    # undirected path 0-1-2-3 and star 9-{10, 11}, both directions given
    g = Csc.from_edges(20, [0, 1, 2, 9, 9, 1, 2, 3, 10, 11], [1, 2, 3, 10, 11, 0, 1, 2, 9, 9])
    b = Bvss.build(g)
    a = b.arrays()
    levels = np.full(20, 0xFFFFFFFF, dtype=np.uint32)
    levels[[0, 1, 2, 3]] = [0, 1, 2, 3]
    deg = np.diff(g.col_ptrs.astype(np.int64))
    assert bench.reached_edges(deg, levels) == 3
    rsets = np.unique(np.array([0, 1, 2, 3]) >> 3)
    rp, ssp = a["real_ptrs"], a["slice_set_ptrs"]
    v_r = int((rp[rsets + 1].astype(np.int64) - rp[rsets]).sum())
    s_r = int((ssp[rp[rsets + 1]].astype(np.int64) - ssp[rp[rsets]].astype(np.int64)).sum())
    assert bench.algorithmic_bytes(a, levels) == 5 * s_r + 12 * v_r + 4 * 4


def test_serving_sweep_is_open_loop_with_per_graph_backlogs():
    """The serving client on a dry-run server: with two result buffers per
    graph, requests beyond them wait in their graph's backlog (arrivals for
    the other graph go on) and every request completes exactly once."""
    from types import SimpleNamespace

    from blest_b200.server import Server

    class DryServer(Server):
        def __init__(self, **kw):
            super().__init__(dry_run=True, **kw)

        def add_graph(self, n):
            return self.add_virtual_graph(n)

    graphs = [("a", None, 1000, np.arange(1, 5, dtype=np.int64), np.arange(4, dtype=np.uint32)),
              ("b", None, 3000, np.arange(1, 5, dtype=np.int64), np.arange(4, dtype=np.uint32))]
    pools = [[np.zeros(n, dtype=np.uint32) for _ in range(2)] for _, _, n, _, _ in graphs]
    args = SimpleNamespace(lanes=1, requests=400, seconds=1.0, always_batch=False)
    rec, = bench.serving_sweep(args, graphs, pools, [4000.0], DryServer)
    assert rec["requests"] == 400 and rec["failed"] == 0 and rec["rejected"] == 0
    assert rec["waited_for_buffer"] > 0 and rec["buffers"] == [2, 2]
    assert rec["jobs"] == sum(rec["jobs_by_kind"].values())
    assert rec["jobs_by_kind"]["bfs"] + rec["requests_by_kind"]["mbfs"] + rec["requests_by_kind"]["cc"] == 400
    assert rec["p99_ms"] >= rec["p50_ms"] > 0
