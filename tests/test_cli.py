"""The `blest -d -g -j -w` driver (C++ over the plugin header
include/blest_kernels.hpp): strict argument handling, caches keyed on
-j/-w, and on the GPU per-source results equal to the oracle."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from blest_b200 import Csc

CLI = Path(__file__).resolve().parents[1] / "blest_b200" / "blest"


def run(*args):
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, timeout=600)


def test_argument_errors():
    r = run("-d", "/tmp", "-g", "x")
    assert r.returncode == 1 and "Missing required option: -j" in r.stderr
    r = run("-d", "/tmp", "-g", "x", "-j", "2", "-w", "8")
    assert r.returncode == 1 and "Invalid value for -j" in r.stderr
    r = run("-d", "/tmp", "-g", "x", "-j", "1", "-w", "abc")
    assert r.returncode == 1 and "Invalid value for -w" in r.stderr
    r = run("-d", "/tmp", "-g", "x", "-j", "1", "-w", "8", "--bogus")
    assert r.returncode == 1 and "Unknown argument" in r.stderr
    r = run("-h")
    assert r.returncode == 0 and "Usage" in r.stderr


def test_mtx_input_and_caches(tmp_path):
    # a small symmetric Matrix Market file
    (tmp_path / "tiny.mtx").write_text(
        "%%MatrixMarket matrix coordinate pattern symmetric\n6 6 5\n2 1\n3 2\n4 3\n6 5\n5 4\n")
    r = run("-d", tmp_path, "-g", "tiny", "-j", "0", "-w", "64", "--sources", "3")
    assert "CSC constructed." in r.stdout
    assert (tmp_path / "tiny_csc.bin").exists()
    assert (tmp_path / "tiny_ordering_j0_w64.bin").exists()
    assert (tmp_path / "tiny.txt").exists()
    c = Csc.load_bin(str(tmp_path / "tiny_csc.bin"))
    assert c.n == 6 and c.nnz == 10
    # second run reuses the caches
    r = run("-d", tmp_path, "-g", "tiny", "-j", "0", "-w", "64")
    assert "CSC read from binary." in r.stdout and "Ordering read from binary." in r.stdout


@pytest.mark.gpu
def test_bfs_results_match_oracle(tmp_path, gpu):
    import oracle as O
    r = run("-d", tmp_path, "-g", "r12", "-j", "1", "-w", "1024", "--gen", "rmat:12:16", "--sources", "8")
    assert r.returncode == 0, r.stderr
    g = Csc.rmat(12, 16, seed=1, permute_seed=1)  # the graph --gen builds (seed 1)
    lines = re.findall(r"Source: (\d+) - Number of levels processed: (\d+) - Total visited: (\d+)", r.stdout)
    assert len(lines) == 8
    for s, levels, visited in lines:
        lv = O.bfs_csc(g.n, g.col_ptrs, g.rows, int(s))
        reached = lv != O.UNREACHED
        assert int(visited) == int(reached.sum())
        assert int(levels) == int(lv[reached].max()) + 1
    r = run("-d", tmp_path, "-g", "r12", "-j", "1", "-w", "1024", "-k", "cc")
    assert r.returncode == 0, r.stderr
    k = int(re.search(r"Number of components identified: (\d+)", r.stdout).group(1))
    assert k == np.unique(O.cc_csc(g.n, g.col_ptrs, g.rows)).size
    r = run("-d", tmp_path, "-g", "r12", "-j", "1", "-w", "1024", "-k", "mbfs")
    assert r.returncode == 0 and "Sources: 8" in r.stdout
