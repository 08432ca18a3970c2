"""The oracle itself: the C restatement against the reference's golden vectors
(tests/golden, produced by the reference's own CPU g2g path) and, when the
reference build is present, against the reference live."""
import os

import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H
from .golden.make_golden import CASES

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_golden(name):
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    wl = CASES[name]()
    E, K, Kb, npts = H.restatement(wl)
    assert abs(E - float(g["E"])) <= 1e-10
    assert np.max(np.abs(K - g["K"])) <= 1e-11
    if wl.open_shell:
        assert np.max(np.abs(Kb - g["Kb"])) <= 1e-11
    assert npts == int(np.sum(g["npts"]))
    E2, F, _ = H.restatement(wl, forces=True)
    assert abs(E2 - float(g["E"])) <= 1e-10
    assert np.max(np.abs(F - g["F"])) <= 1e-11


@pytest.mark.skipif(not os.path.exists(H.REF_LIB), reason="reference build absent")
@pytest.mark.parametrize("seed,natoms,iexch,open_shell", [(101, 9, 9, False), (102, 7, 9, True), (103, 9, 3, False)])
def test_restatement_matches_reference_live(seed, natoms, iexch, open_shell):
    wl = W.small_workload(natoms, seed, iexch, open_shell)
    E_r, K_r, Kb_r = H.reference(wl)
    E, K, Kb, _ = H.restatement(wl)
    assert abs(E - E_r) <= 1e-10
    assert np.max(np.abs(K - K_r)) <= 1e-11
    if open_shell:
        assert np.max(np.abs(Kb - Kb_r)) <= 1e-11


@pytest.mark.skipif(not os.path.exists(H.REF_LIB), reason="reference build absent")
@pytest.mark.parametrize("iexch", [4, 5, 6, 7, 8])
def test_restatement_other_ggas_match_reference_live(iexch):
    """Closed-shell GGAs other than PBE (g2g/pointxc/calc_ggaCS.h:36-262)."""
    wl = W.small_workload(10, 300 + iexch, iexch, False)
    E_r, K_r, _ = H.reference(wl)
    E, K, _, _ = H.restatement(wl)
    assert abs(E - E_r) <= 1e-10
    assert np.max(np.abs(K - K_r)) <= 1e-11


@pytest.mark.skipif(not os.path.exists(H.REF_LIB), reason="reference build absent")
@pytest.mark.parametrize("seed,natoms,iexch,open_shell", [(101, 9, 9, False), (102, 7, 9, True), (104, 6, 2, False),
                                                          (105, 8, 7, False)])
@pytest.mark.parametrize("ctype", [2, 3])
def test_restatement_forces_match_reference_live(seed, natoms, iexch, open_shell, ctype):
    """XC forces (g2g_solve_groups_ types 2 and 3): the restatement's loop
    against the reference's (g2g/cpu/iteration.cpp:213-267, 496-563)."""
    wl = W.small_workload(natoms, seed, iexch, open_shell)
    E_r, F_r = H.reference_forces(wl, ctype)
    E, F, _ = H.restatement(wl, forces=True)
    assert abs(E - E_r) <= 1e-10
    assert np.max(np.abs(F - F_r)) <= 1e-11
    assert np.max(np.abs(F_r)) > 1e-3  # the case has forces to compare


def test_restatement_sampling_partitions_groups():
    """Strided samples of groups add up to the full build (the bounded-sample
    CPU baseline and any group sharding rely on this)."""
    wl = W.small_workload(8, 55, 9, True)
    E, K, Kb, n = H.restatement(wl)
    parts = [H.restatement(wl, first=r, stride=3) for r in range(3)]
    assert abs(sum(p[0] for p in parts) - E) <= 1e-10
    assert np.max(np.abs(sum(p[1] for p in parts) - K)) <= 1e-11
    assert np.max(np.abs(sum(p[2] for p in parts) - Kb)) <= 1e-11
    assert sum(p[3] for p in parts) == n
