"""Shared drivers for the parity tests: run one workload through a g2g-ABI library.

The reference CPU g2g path (oracle/_ref/libg2g_ref.so, built from the reference
sources by oracle/Makefile) is the checker; the product library is
lio_b200/libg2g_b200.so. Both are driven through the same ctypes binding with
the same caller-owned arrays, the way lioamber drives g2g.
"""
import os

import numpy as np

from lio_b200 import workloads as W
from lio_b200.g2g import G2GLibrary, angular_tables

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libg2g_ref.so")
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")

E_TOL = 1e-6   # Ha, |E_xc - E_oracle|
K_TOL = 1e-7   # max |K_xc - K_oracle| over the packed Kohn-Sham matrix

_libs = {}


def lib(path, product):
    key = (path, product)
    if key not in _libs:
        _libs[key] = G2GLibrary(path, product=product)
    return _libs[key]


def bind(L, wl, grid_type=2, options=None):
    e, w = angular_tables(wl.n_ang)
    opts = dict(eai=True)
    if options:
        opts.update(options)
    L.set_options(**opts)
    if wl.n_ang == 194:
        L.bind_workload(wl, {2: (e, w)})
        return 2
    L.bind_workload(wl, {})
    L.set_angular_grid(3, e, w)
    return 3


def subset_tables(n):
    """The first n directions of the 194-point table with their weights scaled to
    sum to 4 pi: a caller table for grid types 0 (n = 50) and 1 (n = 116) that
    both libraries receive alike (parity needs the same table, not a Lebedev one)."""
    e, w = angular_tables(194)
    e, w = np.asfortranarray(e[:n]), np.ascontiguousarray(w[:n])
    return e, w * (4.0 * np.pi / w.sum())


def run_grid_type(L, wl, grid_type, precision=None, options=None):
    """(E, fock, fockb) of one build on grid type 0 (50 directions, radial table
    Nr) or 1 (116 directions, Nr2), the tables passed through g2g_parameter_init_."""
    opts = dict(eai=True)
    if options:
        opts.update(options)
    L.set_options(**opts)
    L.bind_workload(wl, {0: subset_tables(50), 1: subset_tables(116)})
    if precision is not None:
        L.set_precision(precision)
    msg = L.reload_atom_positions(grid_type)
    if msg:
        raise RuntimeError(msg)
    E = L.solve_groups(0)
    return E, L.fock.copy(), L.fockb.copy()


def run(L, wl, calls=1, options=None, precision=None):
    """Returns (E, fock, fockb) after `calls` solves (each accumulates into the
    caller's Fock vectors, like consecutive SCF iterations without a reset)."""
    gt = bind(L, wl, options=options)
    if precision is not None:
        L.set_precision(precision)
    msg = L.reload_atom_positions(gt)
    if msg:
        raise RuntimeError(msg)
    E = None
    for _ in range(calls):
        E = L.solve_groups(0)
    return E, L.fock.copy(), L.fockb.copy()


def run_forces(L, wl, computation_type=2, options=None, precision=None):
    """(E, forces natoms x 3) of one g2g_solve_groups_ type 2 or 3 call."""
    gt = bind(L, wl, options=options)
    if precision is not None:
        L.set_precision(precision)
    msg = L.reload_atom_positions(gt)
    if msg:
        raise RuntimeError(msg)
    return L.solve_forces(computation_type)


def reference_forces(wl, computation_type=2, options=None):
    L = lib(REF_LIB, False)
    L.init()
    out = run_forces(L, wl, computation_type, options=options)
    L.deinit()
    return out


def reference(wl, options=None):
    L = lib(REF_LIB, False)
    L.init()
    out = run(L, wl, options=options)
    L.deinit()
    return out


# ---------------------------------------------------------------- C restatement
import ctypes as C  # noqa: E402


class OracleSystem(C.Structure):
    _fields_ = [("natoms", C.c_int), ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)),
                ("z", C.POINTER(C.c_double)), ("Z", C.POINTER(C.c_int)), ("rm_by_Z", C.POINTER(C.c_double)),
                ("shells_by_Z", C.POINTER(C.c_uint)), ("M", C.c_int), ("nuc", C.POINTER(C.c_int)),
                ("ncont", C.POINTER(C.c_int)), ("a", C.POINTER(C.c_double)), ("c", C.POINTER(C.c_double)),
                ("s_funcs", C.c_int), ("p_funcs", C.c_int), ("d_funcs", C.c_int), ("normalize", C.c_int),
                ("nang", C.c_int), ("ex", C.POINTER(C.c_double)), ("ey", C.POINTER(C.c_double)),
                ("ez", C.POINTER(C.c_double)), ("ew", C.POINTER(C.c_double)),
                ("little_cube_size", C.c_double), ("sphere_radius", C.c_double),
                ("max_function_exponent", C.c_uint), ("min_points_per_cube", C.c_uint),
                ("assign_all_functions", C.c_int), ("remove_zero_weights", C.c_int), ("mincost", C.c_longlong),
                ("iexch", C.c_int), ("open", C.c_int)]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def restatement(wl, first=0, stride=1, options=None, groups=None, forces=False):
    """(E, fock, fockb, npoints) from the C restatement (oracle/liboracle.so);
    with `groups`, only those groups (partition order) are built; with
    forces=True, (E, forces natoms x 3, npoints) of the XC force build."""
    L = _libs.get("oracle")
    if L is None:
        L = C.CDLL(ORACLE_LIB)
        L.oracle_solve_sample.restype = C.c_int
        _libs["oracle"] = L
    opts = dict(lcs=8.0, sr=0.6, mfe=10, mppc=1, aaf=False, rzw=True)
    if options:
        opts.update(options)
    mol, bas = wl.mol, wl.basis
    keep = {}
    keep["x"] = np.ascontiguousarray(mol.pos[:, 0])
    keep["y"] = np.ascontiguousarray(mol.pos[:, 1])
    keep["z"] = np.ascontiguousarray(mol.pos[:, 2])
    keep["Z"] = mol.Z.astype(np.int32)
    keep["rm"] = W.rm_table()
    keep["sh"] = W.shell_tables(wl.n_rad)[1]
    keep["nuc"] = (bas.nuc.astype(np.int32) - 1)
    keep["nc"] = bas.ncont.astype(np.int32)
    keep["a"] = np.ascontiguousarray(bas.a)
    keep["c"] = np.ascontiguousarray(bas.c)
    e, w = angular_tables(wl.n_ang)
    keep["ex"], keep["ey"], keep["ez"] = (np.ascontiguousarray(e[:, k]) for k in range(3))
    keep["ew"] = np.ascontiguousarray(w)
    s = OracleSystem(mol.natom, _dp(keep["x"]), _dp(keep["y"]), _dp(keep["z"]),
                     keep["Z"].ctypes.data_as(C.POINTER(C.c_int)), _dp(keep["rm"]),
                     keep["sh"].ctypes.data_as(C.POINTER(C.c_uint)), bas.M,
                     keep["nuc"].ctypes.data_as(C.POINTER(C.c_int)), keep["nc"].ctypes.data_as(C.POINTER(C.c_int)),
                     _dp(keep["a"]), _dp(keep["c"]), int(bas.nshell[0]), int(bas.nshell[1]) // 3,
                     int(bas.nshell[2]) // 6, 1, len(w), _dp(keep["ex"]), _dp(keep["ey"]), _dp(keep["ez"]),
                     _dp(keep["ew"]), opts["lcs"], opts["sr"], opts["mfe"], opts["mppc"], int(opts["aaf"]),
                     int(opts["rzw"]), 250000, wl.iexch, int(wl.open_shell))
    npk = bas.M * (bas.M + 1) // 2
    fock, fockb = np.zeros(npk), np.zeros(npk)
    E = C.c_double(0)
    npts, ngr = C.c_longlong(0), C.c_longlong(0)
    if wl.open_shell:
        dens = (None, _dp(np.ascontiguousarray(wl.rho_a)), _dp(np.ascontiguousarray(wl.rho_b)))
        keep["ra"], keep["rb"] = wl.rho_a, wl.rho_b
    else:
        r = np.ascontiguousarray(wl.rho)
        keep["r"] = r
        dens = (_dp(r), None, None)
    if forces:
        frc = np.zeros(3 * mol.natom)
        rc = L.oracle_solve_forces(C.byref(s), *dens, _dp(frc), C.byref(E), C.byref(npts), C.byref(ngr))
        assert rc == 0, rc
        return E.value, frc.reshape(3, mol.natom).T.copy(), npts.value
    if groups is not None:
        ids = np.ascontiguousarray(np.asarray(groups, dtype=np.int32))
        rc = L.oracle_solve_subset(C.byref(s), *dens, _dp(fock), _dp(fockb), C.byref(E), C.byref(npts),
                                   C.byref(ngr), ids.ctypes.data_as(C.POINTER(C.c_int)), len(ids))
    else:
        rc = L.oracle_solve_sample(C.byref(s), *dens, _dp(fock), _dp(fockb), C.byref(E), C.byref(npts),
                                   C.byref(ngr), first, stride)
    assert rc == 0, rc
    return E.value, fock, fockb, npts.value


def oracle_result(wl):
    """The checker for a workload: the compiled reference when it can run the
    grid (194 points), else the C restatement."""
    if wl.n_ang == 194 and os.path.exists(REF_LIB):
        return reference(wl)
    E, K, Kb, _ = restatement(wl)
    return E, K, Kb
