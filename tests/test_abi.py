"""The C-ABI library: loads, exports every entry point include/g2g.h declares,
and reports failures through g2g_last_error_ instead of throwing or exiting
(no compute calls here: this runs without a GPU)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from lio_b200 import workloads as W
from lio_b200.g2g import G2GLibrary

from . import helpers as H

PROD = os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so")
HEADER = os.path.join(H.ROOT, "include", "g2g.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(g2g_\w+_)\s*\(", src)))


def test_header_declares_reference_abi():
    names = declared_symbols()
    for ref in ["g2g_init_", "g2g_set_options_", "g2g_parameter_init_", "g2g_reload_atom_positions_",
                "g2g_new_grid_", "g2g_solve_groups_", "g2g_deinit_", "g2g_timer_start_", "g2g_timer_stop_",
                "g2g_timer_pause_", "g2g_timer_sum_start_", "g2g_timer_sum_stop_", "g2g_timer_sum_pause_",
                "g2g_timer_clear_", "g2g_timer_summary_"]:
        assert ref in names


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", PROD], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (g2g_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    lib = C.CDLL(PROD)
    for s in declared_symbols():
        assert hasattr(lib, s)


def test_library_has_no_torch_dependency():
    out = subprocess.run(["ldd", PROD], capture_output=True, text=True).stdout
    assert "libtorch" not in out and "libc10" not in out


def test_errors_are_reported_not_thrown():
    L = G2GLibrary(PROD)
    # solving before any grid exists must set the status, not crash
    e = C.c_double(123.0)
    L.lib.g2g_solve_groups_(C.byref(C.c_uint(0)), C.byref(e), None)
    buf = C.create_string_buffer(256)
    code = L.lib.g2g_last_error_(buf, C.byref(C.c_uint(256)))
    assert code != 0 and b"g2g_solve_groups_" in buf.value
    # reading clears it
    assert L.lib.g2g_last_error_(buf, C.byref(C.c_uint(256))) == 0


def test_invalid_parameters_are_rejected():
    wl = W.small_workload(4, 3, 9, False)
    wl.iexch = 10  # no such functional in the reference (g2g/pointxc/calc_ggaCS.h:264-300)
    L = G2GLibrary(PROD)
    L.set_options()
    with pytest.raises(RuntimeError, match="Iexch"):
        L.bind_workload(wl, {})
    wl.iexch = 9
    wl.basis.ncont[0] = 14  # more primitives than the ABI's 13 (g2g/init.cpp:140-143)
    with pytest.raises(RuntimeError, match="contraction"):
        L.bind_workload(wl, {})


def test_timers_are_callable():
    lib = C.CDLL(PROD)
    name = b"xc_step"
    lib.g2g_timer_sum_start_(name, C.c_uint(len(name)))
    lib.g2g_timer_sum_stop_(name, C.c_uint(len(name)))
    lib.g2g_timer_start_(name, C.c_uint(len(name)))
    lib.g2g_timer_stop_(name, C.c_uint(len(name)))
    lib.g2g_timer_summary_()
    lib.g2g_timer_clear_()


def test_product_library_refuses_to_solve_without_device(monkeypatch):
    """No CPU fallback: on a machine without a CUDA device the grid is built
    (host work) but the solve reports that the device engine is unavailable."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    wl = W.small_workload(4, 3, 9, False)
    L = G2GLibrary(PROD)
    gt = H.bind(L, wl)
    msg = L.reload_atom_positions(gt)
    assert msg and "no CUDA device" in msg
    assert L.partition_stats()["points"] > 0
    with pytest.raises(RuntimeError, match="device"):
        L.solve_groups(0)
