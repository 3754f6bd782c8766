"""The C-ABI library loads and exports every symbol include/*.h declares;
device entry points fail loudly (no CPU fallback) when no GPU is present."""
import ctypes
import subprocess

import numpy as np
import pytest

from blest_b200 import _lib as L
from blest_b200 import BlestError, Bvss, Csc


def test_exports_every_declared_symbol():
    names = L.declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(L.lib, n)]
    assert not missing, missing


def test_exported_symbols_via_nm():
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for n in L.declared_symbols():
        assert n in exported, n


def test_version_and_error_string():
    assert b"sm_100a" in L.lib.blest_version()
    rc = L.fn["blest_csc_load_bin"](b"/nonexistent/x_csc.bin", ctypes.byref(ctypes.c_void_p()))
    assert rc == L.ERR_IO
    assert b"cannot open" in L.lib.blest_last_error()


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_no_gpu_fails_loudly():
    with pytest.raises(BlestError) as e:
        L.call("blest_init", 0)
    assert e.value.code == L.ERR_NO_DEVICE
    c = Csc.rmat(6, 4, seed=1)
    b = Bvss.build(c)
    from blest_b200.graph import Graph
    with pytest.raises(BlestError) as e:
        Graph(b, c)
    assert e.value.code == L.ERR_NO_DEVICE


def test_null_arguments_are_rejected():
    assert L.fn["blest_bfs"](None, 0, None, None, 0, None, None) == L.ERR_INVALID_ARG
    assert L.fn["blest_csc_view_get"](None, None) == L.ERR_INVALID_ARG
    lab = np.zeros(3, dtype=np.uint32)
    assert L.fn["blest_cc_relabel_dense"](lab.ctypes.data_as(L.P(L.u32)), 3, None, None) == L.ERR_INVALID_ARG
