"""The failure path of the pipelined tensor-core kernels, on purpose and without
a GPU fault.

Every wait of those kernels on an mbarrier is bounded. When a wait runs out,
the kernel records the failure, lets its copies in flight land, frees its TMEM
and returns; the host then reports an error through g2g_last_error_. The
reference has no such path: a failed build ends the process with exit(1)
(g2g/partition.cpp:584-590). Here a self-test kernel whose producer stops
early (it arms and sends one of two ring stages) makes the consumer's second
wait run out after a short poll limit; the test checks the status and the
message, and that the next XC build on the same GPU is still correct.
"""
import ctypes as C
import os

import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H

pytestmark = pytest.mark.gpu

PROD = os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so")


def test_bounded_wait_runs_out_and_next_build_is_correct():
    L = H.lib(PROD, True)
    L.lib.g2g_selftest_bounded_wait_.restype = C.c_int
    L.check("before", raise_=False)  # clear any earlier status
    ms = C.c_double(-1.0)
    rc = L.lib.g2g_selftest_bounded_wait_(C.byref(C.c_uint(1 << 16)), C.byref(ms))
    assert rc == 1, rc
    buf = C.create_string_buffer(512)
    code = L.lib.g2g_last_error_(buf, C.byref(C.c_uint(512)))
    assert code == 3
    assert b"timed out" in buf.value
    assert 0.0 < ms.value < 10_000.0  # the kernel returned on its own
    # the context is usable: a tensor-core build right after is within the parity tolerances
    wl = W.small_workload(10, 31, 9, True)
    E, K, Kb = H.run(L, wl, precision=1)
    E_ref, K_ref, Kb_ref = H.oracle_result(wl)
    assert abs(E - E_ref) <= H.E_TOL
    assert max(np.max(np.abs(K - K_ref)), np.max(np.abs(Kb - Kb_ref))) <= H.K_TOL
