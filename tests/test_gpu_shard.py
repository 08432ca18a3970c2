"""Sharded builds on one GPU: the shares of g2g_set_shard_(rank, world) built one
after another in one process add up to the whole build (E_xc and the
Kohn-Sham matrices), in both forms."""
import ctypes as C
import os

import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H

pytestmark = pytest.mark.gpu

PROD = os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so")


def _share(L, wl, rank, world, precision):
    L.lib.g2g_set_shard_(C.byref(C.c_int(rank)), C.byref(C.c_int(world)))
    try:
        return H.run(L, wl, precision=precision)
    finally:
        L.lib.g2g_set_shard_(C.byref(C.c_int(0)), C.byref(C.c_int(1)))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("world", [2, 3])
def test_shards_add_up_to_the_whole_build(precision, world):
    wl = W.small_workload(14, 77, 9, True, n_ang=302)
    L = H.lib(PROD, True)
    E, K, Kb = _share(L, wl, 0, 1, precision)
    Es, Ks, Kbs = 0.0, np.zeros_like(K), np.zeros_like(Kb)
    for r in range(world):
        e, k, kb = _share(L, wl, r, world, precision)
        Es += e
        Ks += k
        Kbs += kb
    assert abs(Es - E) <= 1e-10
    assert np.max(np.abs(Ks - K)) <= 1e-12
    assert np.max(np.abs(Kbs - Kb)) <= 1e-12
