"""Grid build with the Becke weights on the GPU: the partition (points,
weights, function lists) equals the reference's bit for bit, as the host
build does (tests/test_partition.py), and equals the host build."""
import os

import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H
from .test_partition import PROD, assert_same, reference_groups

pytestmark = pytest.mark.gpu


def product_groups(wl, device_weights, options=None):
    L = H.lib(PROD, True)
    gt = H.bind(L, wl, options=options)
    L.set_device_weights(device_weights)
    msg = L.reload_atom_positions(gt)
    L.set_device_weights(True)
    assert not msg, msg
    out = {}
    for g in range(L.num_groups()):
        d = L.partition_group(g)
        out[tuple(sorted(map(tuple, d["ids"].tolist())))] = d
    return out


@pytest.mark.skipif(not os.path.exists(H.REF_LIB), reason="reference build absent")
@pytest.mark.parametrize("make,options", [
    (lambda: W.config(1), None),
    (lambda: W.small_workload(16, 7, 9, False), None),
    (lambda: W.small_workload(12, 11, 9, True), dict(lcs=5.0, sr=0.4)),
    (lambda: W.small_workload(9, 17, 9, False), dict(rzw=False)),
    (lambda: W.small_workload(8, 19, 3, False), dict(aaf=True, sr=0.0)),
], ids=["cfg1", "pbe16", "small-cubes", "keep-zero-weights", "all-functions-no-spheres"])
def test_device_weights_bit_exact_vs_reference(make, options):
    wl = make()
    assert_same(product_groups(wl, True, options), reference_groups(wl, options))


def test_device_weights_equal_host_weights_256_atoms():
    wl = W.config(3)
    dev = product_groups(wl, True)
    host = product_groups(wl, False)
    assert_same(dev, host)
    assert sum(d["meta"][0] for d in dev.values()) == 2867542
