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


def test_documented_host_programs_compile_and_link(tmp_path):
    """A C++ driver on the plugin classes (the reference's Benchmark flow)
    and a C program on the multi-graph plan API, as a user of the library
    writes them, compile against include/ and link against the library."""
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    inc, libdir = root / "include", root / "blest_b200"
    cpp = tmp_path / "driver.cpp"
    cpp.write_text('''
#include <vector>
#include "blest_kernels.hpp"
int main() {
    blest_csc* csc = nullptr;
    if (blest_csc_read_mtx_auto("graph.mtx", &csc) != BLEST_OK) return 1;
    blest_csc_view v;
    blest_csc_view_get(csc, &v);
    blest_order_params op{BLEST_ORDER_AUTO, 1, 65536, 0, 1, 0};
    std::vector<uint32_t> inv(v.n);
    blest_csc_reorder(csc, &op, inv.data());
    blest_bvss* bvss = nullptr;
    blest_bvss_build(csc, -1, &bvss);
    blest_init(0);
    blest_b200::DeviceGraph graph(bvss, csc);
    blest_b200::B200BFSKernel kernel(&graph);
    blest_b200::BFSResult r = kernel.run(inv[0]);
    delete[] r.levels;
    return 0;
}
''')
    c = tmp_path / "plan.c"
    c.write_text('''
#include "blest.h"
int main(void) {
    blest_mbfs_item items[1] = {{0, 0, 0, 0}};
    blest_mbfs_params mp = {32, 0, 0, 0.0625, 0};
    blest_mbfs_plan* plan = 0;
    blest_mbfs_stats st;
    blest_mbfs_plan_info info;
    if (blest_mbfs_plan_create(items, 1, &mp, 0, &plan) != BLEST_OK) return 1;
    blest_mbfs_plan_info_get(plan, &info);
    blest_mbfs_plan_run(plan, &st);
    blest_mbfs_plan_destroy(plan);
    return 0;
}
''')
    for cmd in (["g++", "-std=c++17", f"-I{inc}", str(cpp), f"-L{libdir}", "-lblest_b200", "-o", str(tmp_path / "d")],
                ["gcc", "-std=c11", f"-I{inc}", str(c), f"-L{libdir}", "-lblest_b200", "-o", str(tmp_path / "p")]):
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
