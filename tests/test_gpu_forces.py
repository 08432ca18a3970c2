"""XC nuclear forces on the device (g2g_solve_groups_ types 2 and 3) against
the reference CPU g2g path (194-point grids) and the C restatement (302).

The reference adds each atom's XC force, -sum_p f_p sum_(i on atom) w_i grad F_i
with w_i = 2 sum_j P_ij F_j (g2g/cpu/iteration.cpp:213-267, open shell
496-563), into the caller's natoms x 3 array and leaves the Kohn-Sham vectors
alone. The device evaluates the same sum in FP64 from the factors of its build;
with the tensor-core form those factors carry that form's density error.
"""
import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H

pytestmark = pytest.mark.gpu

F_TOL = 1e-7  # Hartree/bohr, max |F - F_oracle| over atoms and axes

CASES = [
    ("cfg1-lda-vwn", lambda: W.config(1)),
    ("pbe-closed-12", lambda: W.small_workload(12, 21, 9, False)),
    ("pbe-open-10", lambda: W.small_workload(10, 31, 9, True)),
    ("lda-gl-8", lambda: W.small_workload(8, 41, 2, False)),
]


def _product():
    return H.lib(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("ctype", [2, 3])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_forces_match_reference(name, make, ctype, precision):
    wl = make()
    E_ref, F_ref = H.reference_forces(wl, ctype)
    P = _product()
    E, F = H.run_forces(P, wl, ctype, precision=precision)
    assert F.shape == F_ref.shape == (wl.mol.natom, 3)
    assert np.max(np.abs(F_ref)) > 1e-3
    assert abs(E - E_ref) <= H.E_TOL, (E, E_ref)
    assert np.max(np.abs(F - F_ref)) <= F_TOL, np.max(np.abs(F - F_ref))
    # no Kohn-Sham update for types 2 and 3
    assert not np.any(P.fock) and not np.any(P.fockb)
    print(name, ctype, precision, E - E_ref, np.max(np.abs(F - F_ref)))


@pytest.mark.parametrize("precision", [0, 1])
def test_forces_match_restatement_302(precision):
    wl = W.config(2)  # 64 atoms, closed-shell PBE, 40 x 302
    E_ref, F_ref, npts = H.restatement(wl, forces=True)
    P = _product()
    E, F = H.run_forces(P, wl, 2, precision=precision)
    assert P.partition_stats()["points"] == npts
    assert abs(E - E_ref) <= H.E_TOL, (E, E_ref)
    assert np.max(np.abs(F - F_ref)) <= F_TOL, np.max(np.abs(F - F_ref))
    print("cfg2", precision, E - E_ref, np.max(np.abs(F - F_ref)), np.max(np.abs(F_ref)))


def test_forces_then_fock_build():
    """A force call between Fock builds leaves the next build's result intact
    (the force path shares the density upload and factor buffers)."""
    wl = W.small_workload(10, 31, 9, True)
    P = _product()
    E0, K0, Kb0 = H.run(P, wl, precision=1)
    P.fock[:] = 0.0
    P.fockb[:] = 0.0
    P.solve_forces(2)
    E1 = P.solve_groups(0)
    assert abs(E1 - E0) <= 1e-12
    assert np.max(np.abs(P.fock - K0)) <= 1e-12
    assert np.max(np.abs(P.fockb - Kb0)) <= 1e-12
