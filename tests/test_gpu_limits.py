"""Limits of the tensor-core form that the engine enforces on the host.

The Kohn-Sham contraction sums int8 digit products over a point group's points
in int32 level accumulators, exact only up to 87,296 padded points per group.
A grid whose cubes are large enough to hold more (here one cube for the whole
molecule, through little_cube_size) must be refused with a clear error, before
any kernel runs, while the FP64 form still builds it."""
import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H


@pytest.mark.gpu
def test_tensor_core_refuses_a_group_above_its_accumulator_limit():
    wl = W.small_workload(24, 5, 9, False)
    L = H.lib(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)
    gt = H.bind(L, wl, options=dict(lcs=1000.0, sr=0.0))  # every point in one cube
    L.set_precision(1)
    msg = L.reload_atom_positions(gt)
    assert not msg, msg
    st = L.partition_stats()
    big = max(L.partition_group(g)["meta"][0] for g in range(st["groups"]))
    assert big > 87296, big
    with pytest.raises(RuntimeError, match="exceeds its limit"):
        L.solve_groups(0)
    L.set_precision(0)
    E = L.solve_groups(0)
    assert np.isfinite(E)
    L.deinit()
