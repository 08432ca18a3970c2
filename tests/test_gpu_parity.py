"""FP64 device path vs the reference CPU g2g path (E_xc and the packed Kohn-Sham matrix)."""
import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H

pytestmark = pytest.mark.gpu

CASES = [
    ("cfg1-lda-vwn", lambda: W.config(1)),
    ("pbe-closed-12", lambda: W.small_workload(12, 21, 9, False)),
    ("pbe-open-10", lambda: W.small_workload(10, 31, 9, True)),
    ("lda-gl-8", lambda: W.small_workload(8, 41, 2, False)),
    ("slater-8", lambda: W.small_workload(8, 43, 1, False)),
    ("p86-9", lambda: W.small_workload(9, 205, 4, False)),
    ("b88-p86-9", lambda: W.small_workload(9, 206, 5, False)),
    ("b88-vwn-8", lambda: W.small_workload(8, 207, 6, False)),
    ("blyp-10", lambda: W.small_workload(10, 208, 7, False)),
    ("p86-lyp-9", lambda: W.small_workload(9, 209, 8, False)),
    ("blyp-open-8", lambda: W.small_workload(8, 210, 7, True)),  # open shell: PBE, as the reference
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_fp64_matches_reference(name, make):
    wl = make()
    E_ref, K_ref, Kb_ref = H.reference(wl)
    P = H.lib(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)
    E, K, Kb = H.run(P, wl, precision=0)
    assert abs(E - E_ref) <= H.E_TOL, (E, E_ref)
    assert np.max(np.abs(K - K_ref)) <= H.K_TOL
    if wl.open_shell:
        assert np.max(np.abs(Kb - Kb_ref)) <= H.K_TOL
    print(name, E, E_ref, abs(E - E_ref), np.max(np.abs(K - K_ref)))


# The 302-point configurations cannot run on the compiled reference (its angular
# tables are compile-time), so their checker is the C restatement, which the
# CPU tests pin to the reference on the 194-point grid.
BIG = [("cfg2-302-closed-pbe", lambda: W.config(2)), ("cfg3-302-open-pbe", lambda: W.config(3))]


@pytest.mark.parametrize("name,make", BIG, ids=[c[0] for c in BIG])
def test_fp64_matches_restatement_302(name, make):
    wl = make()
    E_ref, K_ref, Kb_ref, npts = H.restatement(wl)
    P = H.lib(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)
    E, K, Kb = H.run(P, wl, precision=0)
    assert P.partition_stats()["points"] == npts
    assert abs(E - E_ref) <= H.E_TOL, (E, E_ref)
    assert np.max(np.abs(K - K_ref)) <= H.K_TOL
    if wl.open_shell:
        assert np.max(np.abs(Kb - Kb_ref)) <= H.K_TOL
    print(name, npts, E, E_ref, abs(E - E_ref), np.max(np.abs(K - K_ref)))


# Tensor-core form (precision 1): the density contraction runs as int8
# Ozaki-slice products on tcgen05; same tolerances as the FP64 form.
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_tensor_core_matches_reference(name, make):
    wl = make()
    E_ref, K_ref, Kb_ref = H.reference(wl)
    P = H.lib(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)
    E, K, Kb = H.run(P, wl, precision=1)
    print(name, "tc", E, E_ref, abs(E - E_ref), np.max(np.abs(K - K_ref)))
    assert abs(E - E_ref) <= H.E_TOL, (E, E_ref)
    assert np.max(np.abs(K - K_ref)) <= H.K_TOL
    if wl.open_shell:
        assert np.max(np.abs(Kb - Kb_ref)) <= H.K_TOL


@pytest.mark.parametrize("name,make", BIG, ids=[c[0] for c in BIG])
def test_tensor_core_matches_restatement_302(name, make):
    wl = make()
    E_ref, K_ref, Kb_ref, npts = H.restatement(wl)
    P = H.lib(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)
    E, K, Kb = H.run(P, wl, precision=1)
    print(name, "tc", npts, E, E_ref, abs(E - E_ref), np.max(np.abs(K - K_ref)))
    assert abs(E - E_ref) <= H.E_TOL, (E, E_ref)
    assert np.max(np.abs(K - K_ref)) <= H.K_TOL
    if wl.open_shell:
        assert np.max(np.abs(Kb - Kb_ref)) <= H.K_TOL


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("grid_type", [0, 1])
def test_grid_types_0_1_match_reference(grid_type, precision):
    """Grid types 0 and 1 (their own radial and angular tables) through both forms."""
    wl = W.small_workload(10, 23, 9, True)
    R = H.lib(H.REF_LIB, False)
    R.init()
    E_ref, K_ref, Kb_ref = H.run_grid_type(R, wl, grid_type)
    R.deinit()
    P = H.lib(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)
    E, K, Kb = H.run_grid_type(P, wl, grid_type, precision=precision)
    assert abs(E - E_ref) <= H.E_TOL, (E, E_ref)
    assert np.max(np.abs(K - K_ref)) <= H.K_TOL
    assert np.max(np.abs(Kb - Kb_ref)) <= H.K_TOL


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("grid_type", [0, 1, 2])
def test_lio_tables_match_reference(grid_type, precision):
    """Builds on lioamber's own angular tables (lioamber/grid.f90:39-476, as
    tests/golden/make_lio_tables.py evaluates them), grid types 0, 1, 2."""
    from .test_partition import lio_tables

    wl = W.small_workload(12, 29, 9, True)
    tables = lio_tables()

    def build(path, product):
        L = H.lib(path, product)
        if not product:
            L.init()
        L.set_options(eai=True)
        L.bind_workload(wl, tables)
        if product:
            L.set_precision(precision)
        msg = L.reload_atom_positions(grid_type)
        assert not msg, msg
        E = L.solve_groups(0)
        out = (E, L.fock.copy(), L.fockb.copy())
        if not product:
            L.deinit()
        return out

    E_ref, K_ref, Kb_ref = build(H.REF_LIB, False)
    E, K, Kb = build(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)
    assert abs(E - E_ref) <= H.E_TOL, (E, E_ref)
    assert np.max(np.abs(K - K_ref)) <= H.K_TOL
    assert np.max(np.abs(Kb - Kb_ref)) <= H.K_TOL
