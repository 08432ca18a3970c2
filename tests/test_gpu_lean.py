"""Lean tensor-core form (g2g_set_lean_): the blocked FP64 basis is released once
the operands are built, the Kohn-Sham kernels form F from the per-shell radial
sums, and forces rebuild the blocked basis for their call.

* E_xc and K against the reference CPU g2g path (194-point grids) and the C
  restatement (the 64-atom 302-point case), at the parity tolerances.
* Against the form that keeps the blocked basis: the radial-sum F values equal
  k_basis's up to the order of one product, so E and K agree to ~1e-12.
* Forces equal the non-lean form's and match the reference.
"""
import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H

pytestmark = pytest.mark.gpu

SAME = 1e-11  # lean vs kept basis: F differs only in product order (a few ulp)

CASES = [
    ("cfg1-lda-vwn", lambda: W.config(1)),
    ("pbe-closed-12", lambda: W.small_workload(12, 21, 9, False)),
    ("pbe-open-10", lambda: W.small_workload(10, 31, 9, True)),
    ("blyp-open-8", lambda: W.small_workload(8, 210, 7, True)),
]


def product():
    return H.lib(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)


def lean_run(wl, forces=False):
    P = product()
    P.set_lean(True)
    try:
        return H.run_forces(P, wl, precision=1) if forces else H.run(P, wl, precision=1)
    finally:
        P.set_lean(False)


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_lean_matches_reference_and_kept_basis(name, make):
    wl = make()
    E_ref, K_ref, Kb_ref = H.reference(wl)
    E1, K1, Kb1 = H.run(product(), wl, precision=1)
    E, K, Kb = lean_run(wl)
    print(name, "lean", E, E_ref, abs(E - E_ref), np.max(np.abs(K - K_ref)), np.max(np.abs(K - K1)))
    assert abs(E - E_ref) <= H.E_TOL and np.max(np.abs(K - K_ref)) <= H.K_TOL
    assert abs(E - E1) <= SAME and np.max(np.abs(K - K1)) <= SAME
    if wl.open_shell:
        assert np.max(np.abs(Kb - Kb_ref)) <= H.K_TOL and np.max(np.abs(Kb - Kb1)) <= SAME


def test_lean_matches_restatement_302():
    wl = W.config(2)
    E_ref, K_ref, _, npts = H.restatement(wl)
    E, K, _ = lean_run(wl)
    print("cfg2 lean", npts, E, E_ref, abs(E - E_ref), np.max(np.abs(K - K_ref)))
    assert abs(E - E_ref) <= H.E_TOL and np.max(np.abs(K - K_ref)) <= H.K_TOL


@pytest.mark.parametrize("name,make", CASES[1:3], ids=[c[0] for c in CASES[1:3]])
def test_lean_forces(name, make):
    wl = make()
    E_ref, F_ref = H.reference_forces(wl)
    E1, F1 = H.run_forces(product(), wl, precision=1)
    E, F = lean_run(wl, forces=True)
    print(name, "lean forces", np.max(np.abs(F - F_ref)), np.max(np.abs(F - F1)))
    assert np.max(np.abs(F - F1)) <= SAME
    assert np.max(np.abs(F - F_ref)) <= 1e-7  # the force tolerance of the other force tests
