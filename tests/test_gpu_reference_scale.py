"""The 64- and 256-atom molecules against the reference itself.

The 302-point configurations can only be checked against the C restatement
(the reference's angular tables are compile-time), so here the same two
molecules run on their 40 x 194 grids through the compiled reference CPU g2g
path (oracle/_ref/libg2g_ref.so) and through the product, in both forms:

* the grid partition is the same bit for bit: groups keyed by the multiset of
  their (atom, shell, point) ids, weights compared bitwise, function lists
  equal (the product's Becke weights run on the GPU);
* |dE_xc| <= 1e-6 Ha and max |dK| <= 1e-7 over the packed Kohn-Sham matrix
  (both spins for the open-shell molecule).

Reference call path: g2g_reload_atom_positions_ -> g2g_solve_groups_(0)
(g2g/init.cpp:282-391 -> g2g/partition.cpp:426-591).
"""
import os

import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H
from .test_partition import assert_same, product_groups, reference_groups

pytestmark = pytest.mark.gpu

PROD = os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so")


def molecule_194(n):
    """The 64-atom (closed-shell PBE) and 256-atom (open-shell PBE) molecules
    of the single-molecule workloads, on 40 radial x 194 angular points."""
    if n == 64:
        return W.make_workload("cfg2 molecule, 40x194", {"C": 16, "N": 4, "O": 4, "H": 40}, 14.0, 2000, 9, False,
                               194, 40, nocc=62)
    return W.make_workload("cfg3 molecule, 40x194", {"C": 64, "N": 16, "O": 16, "H": 160}, 22.0, 3000, 9, True,
                           194, 40)


_ref_cache = {}


def reference_result(n):
    if n not in _ref_cache:
        _ref_cache[n] = H.reference(molecule_194(n))
    return _ref_cache[n]


@pytest.mark.skipif(not os.path.exists(H.REF_LIB), reason="reference build absent")
@pytest.mark.parametrize("n", [64, 256])
def test_partition_bit_exact_vs_reference_at_scale(n):
    wl = molecule_194(n)
    prod, ref = product_groups(wl), reference_groups(wl)
    assert len(prod) == len(ref) > 0
    assert_same(prod, ref)


@pytest.mark.skipif(not os.path.exists(H.REF_LIB), reason="reference build absent")
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "tensor-core"])
@pytest.mark.parametrize("n", [64, 256])
def test_build_matches_reference_at_scale(n, precision):
    wl = molecule_194(n)
    E_ref, K_ref, Kb_ref = reference_result(n)
    P = H.lib(PROD, True)
    E, K, Kb = H.run(P, wl, precision=precision)
    dE = abs(E - E_ref)
    dK = float(np.max(np.abs(K - K_ref)))
    if wl.open_shell:
        dK = max(dK, float(np.max(np.abs(Kb - Kb_ref))))
    print(f"{n} atoms, 40x194, precision {precision}: E {E:.10f} ref {E_ref:.10f} |dE| {dE:.2e} max|dK| {dK:.2e}")
    assert dE <= H.E_TOL, (E, E_ref)
    assert dK <= H.K_TOL
