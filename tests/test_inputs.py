"""Host-side inputs: the Lebedev tables solved here, packed-storage conventions
and the synthetic workloads."""
import numpy as np
import pytest

from lio_b200 import lebedev
from lio_b200 import workloads as W
from lio_b200.g2g import angular_tables


@pytest.mark.parametrize("n,degree", [(194, 23), (302, 29)])
def test_lebedev_tables_exact_to_their_degree(n, degree):
    e, w = angular_tables(n)
    assert e.shape == (n, 3)
    assert np.allclose(np.sum(e * e, axis=1), 1.0, atol=1e-15)
    assert abs(np.sum(w) - 4 * np.pi) < 1e-12
    assert np.all(w > 0)
    assert lebedev.max_moment_error(np.asarray(e), w, degree) < 1e-12
    # and not exact one even degree higher (they are the minimal grids of that order)
    assert lebedev.max_moment_error(np.asarray(e), w, degree + 2) > 1e-6
    # octahedral symmetry: closed under coordinate sign flips
    pts = {tuple(np.round(p, 10)) for p in np.asarray(e)}
    for p in list(pts)[:20]:
        assert tuple(np.round(-np.array(p), 10) + 0.0) in pts


def test_packed_storage_roundtrip_and_doubling():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((7, 7))
    S = A + A.T
    v = W.pack_lower(S, double_offdiag=False)
    assert np.array_equal(W.unpack_lower(v, 7), S)
    vd = W.pack_lower(S, double_offdiag=True)
    M = 7
    for i in range(M):
        for j in range(i, M):
            k = i * M - i * (i - 1) // 2 + (j - i)  # g2g/partition.cpp:64-66
            assert vd[k] == (S[i, j] if i == j else 2 * S[i, j])


def test_workload_conventions():
    wl = W.config(1)
    assert wl.mol.natom == 8 and sorted(wl.mol.symbols) == ["C", "C"] + ["H"] * 6
    assert wl.basis.M == 2 * 15 + 6 * 5
    s, p3, d6 = wl.basis.nshell
    assert s + p3 + d6 == wl.basis.M
    assert np.all(wl.basis.lmom[:s] == 0) and np.all(wl.basis.lmom[s:s + p3] == 1) and np.all(wl.basis.lmom[s + p3:] == 2)
    # atoms at least 0.9 A apart
    d = np.linalg.norm(wl.mol.pos[:, None] - wl.mol.pos[None], axis=-1) * W.BOHR_ANGSTROM
    assert np.min(d[np.triu_indices(8, 1)]) >= 0.9
    # P = 2 C C^T with orthonormal C: idempotent up to the factor 2
    P = W.unpack_lower(wl.rho, wl.basis.M)
    P[~np.eye(wl.basis.M, dtype=bool)] /= 2
    assert np.allclose(P @ P, 2 * P, atol=1e-12)
    assert abs(np.trace(P) - 2 * 9) < 1e-12
    o = W.small_workload(6, 3, 9, True)
    assert np.allclose(o.rho, o.rho_a + o.rho_b)
