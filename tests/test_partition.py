"""Host grid partition of the product library vs the reference, bit for bit
(runs without a GPU: the partition is host work and stays inspectable through
g2g_partition_group_ even when no device is present)."""
import os

import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H
from .golden.make_golden import CASES

PROD = os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so")
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def product_groups(wl, options=None):
    L = H.lib(PROD, True)
    gt = H.bind(L, wl, options=options)
    L.reload_atom_positions(gt)  # without a GPU this reports the missing device after building the partition
    out = {}
    for g in range(L.num_groups()):
        d = L.partition_group(g)
        out[tuple(sorted(map(tuple, d["ids"].tolist())))] = d
    return out


def reference_groups(wl, options=None):
    L = H.lib(H.REF_LIB, False)
    L.init()
    gt = H.bind(L, wl, options=options)
    L.reload_atom_positions(gt)
    out = {}
    for g in range(L.num_groups(ref=True)):
        d = L.partition_group(g, ref=True)
        out[tuple(sorted(map(tuple, d["ids"].tolist())))] = d
    L.deinit()
    return out


def assert_same(a, b):
    assert set(a) == set(b)
    for k in a:
        x, y = a[k], b[k]
        ix, iy = np.lexsort(x["ids"].T[::-1]), np.lexsort(y["ids"].T[::-1])
        assert x["meta"][:6] == y["meta"][:6]
        assert np.array_equal(x["funcs"], y["funcs"])
        assert np.array_equal(x["xyzw"][ix].view(np.uint64), y["xyzw"][iy].view(np.uint64))  # bitwise


@pytest.mark.skipif(not os.path.exists(H.REF_LIB), reason="reference build absent")
@pytest.mark.parametrize("make,options", [
    (lambda: W.config(1), None),
    (lambda: W.small_workload(16, 7, 9, False), None),
    (lambda: W.small_workload(12, 11, 9, True), dict(lcs=5.0, sr=0.4)),
    (lambda: W.small_workload(10, 13, 9, False), dict(mfe=12, mppc=20)),
    (lambda: W.small_workload(9, 17, 9, False), dict(rzw=False)),
    (lambda: W.small_workload(8, 19, 3, False), dict(aaf=True, sr=0.0)),
], ids=["cfg1", "pbe16", "small-cubes", "mfe12-mppc20", "keep-zero-weights", "all-functions-no-spheres"])
def test_partition_bit_exact_vs_reference(make, options):
    wl = make()
    assert_same(product_groups(wl, options), reference_groups(wl, options))


@pytest.mark.parametrize("name", sorted(CASES))
def test_partition_matches_golden_summary(name):
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    groups = product_groups(CASES[name]())
    npts = np.array([d["meta"][0] for d in groups.values()])
    nfun = np.array([d["meta"][5] for d in groups.values()])
    wsum = np.array([float(np.sum(d["xyzw"][:, 3])) for d in groups.values()])
    o = np.lexsort((wsum, nfun, npts))
    assert np.array_equal(npts[o], g["npts"]) and np.array_equal(nfun[o], g["nfun"])
    assert np.array_equal(wsum[o], g["wsum"])


@pytest.mark.skipif(not os.path.exists(H.REF_LIB), reason="reference build absent")
@pytest.mark.parametrize("grid_type", [0, 1])
def test_partition_bit_exact_vs_reference_grid_types_0_1(grid_type):
    """Grid types 0 (radial table Nr, 50 directions) and 1 (Nr2, 116) select
    their tables as g2g/init.cpp:238-266 does."""
    wl = W.small_workload(10, 23, 9, False)
    tables = {0: H.subset_tables(50), 1: H.subset_tables(116)}

    def groups(path, product):
        L = H.lib(path, product)
        if not product:
            L.init()
        L.set_options(eai=True)
        L.bind_workload(wl, tables)
        L.reload_atom_positions(grid_type)
        out = {}
        for g in range(L.num_groups(ref=not product)):
            d = L.partition_group(g, ref=not product)
            out[tuple(sorted(map(tuple, d["ids"].tolist())))] = d
        if not product:
            L.deinit()
        return out

    prod, ref = groups(PROD, True), groups(H.REF_LIB, False)
    assert_same(prod, ref)
    assert len(prod) > 0


def lio_tables():
    """lioamber's own angular tables for grid types 0, 1, 2 (50, 116, 194
    directions), evaluated from lioamber/grid.f90:39-476 by
    tests/golden/make_lio_tables.py."""
    g = np.load(os.path.join(GOLD, "lio_angular_tables.npz"))
    return {t: (np.asfortranarray(g[f"e{t}"]), np.ascontiguousarray(g[f"w{t}"])) for t in (0, 1, 2)}


@pytest.mark.skipif(not os.path.exists(H.REF_LIB), reason="reference build absent")
@pytest.mark.parametrize("grid_type", [0, 1, 2])
def test_partition_bit_exact_vs_reference_lio_tables(grid_type):
    """The tables lioamber actually passes (not this project's solved Lebedev
    grids), through g2g_parameter_init_ to both libraries."""
    wl = W.small_workload(12, 29, 9, True)
    tables = lio_tables()

    def groups(path, product):
        L = H.lib(path, product)
        if not product:
            L.init()
        L.set_options(eai=True)
        L.bind_workload(wl, tables)
        L.reload_atom_positions(grid_type)
        out = {}
        for g in range(L.num_groups(ref=not product)):
            d = L.partition_group(g, ref=not product)
            out[tuple(sorted(map(tuple, d["ids"].tolist())))] = d
        if not product:
            L.deinit()
        return out

    prod, ref = groups(PROD, True), groups(H.REF_LIB, False)
    assert len(prod) > 0
    assert_same(prod, ref)
