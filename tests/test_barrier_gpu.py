"""The bounded grid barrier's failure path, made to run out on purpose
without faulting or hanging the GPU: a cooperative launch whose barrier
expects one block more than it has can never complete, so every wait must
give up after its (short) limit and report BLEST_ERR_BARRIER_TIMEOUT; the
device must stay usable afterwards."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from blest_b200 import Csc, Graph
from blest_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _run(blocks, missing, timeout_ns, rounds):
    secs = C.c_double(-1.0)
    rc = L.fn["blest_selftest_barrier"](blocks, missing, timeout_ns, rounds, C.byref(secs))
    return rc, secs.value


def test_barrier_completes_when_every_block_arrives(gpu):
    rc, secs = _run(148, 0, 1_000_000_000, 64)
    assert rc == L.OK, L.lib.blest_last_error()
    assert 0 <= secs < 1.0


@pytest.mark.parametrize("blocks", [1, 148, 296])
def test_barrier_wait_runs_out_and_the_device_stays_usable(gpu, blocks):
    # 1 ms limit: the launch must end by itself well within a second
    rc, secs = _run(blocks, 1, 1_000_000, 4)
    assert rc == L.ERR_BARRIER_TIMEOUT
    assert "timed out" in L.lib.blest_last_error().decode()
    assert 0 <= secs < 0.5
    # the context is intact: a full BFS still matches the oracle
    csc = Csc.rmat(10, 8, seed=2, permute_seed=1)
    csc.reorder("jaccard", window=256)
    from blest_b200 import Bvss
    g = Graph(Bvss.build(csc), csc.transpose())
    lv, _, _ = g.bfs(5)
    np.testing.assert_array_equal(lv, O.bfs_csc(csc.n, csc.col_ptrs, csc.rows, 5))


def test_barrier_selftest_rejects_bad_arguments(gpu):
    assert _run(0, 0, 1_000_000, 1)[0] == L.ERR_INVALID_ARG
    assert _run(4, 0, 10, 1)[0] == L.ERR_INVALID_ARG
    assert _run(1 << 20, 0, 1_000_000, 1)[0] == L.ERR_INVALID_ARG
