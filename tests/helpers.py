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


def reference(wl, options=None):
    L = lib(REF_LIB, False)
    L.init()
    out = run(L, wl, options=options)
    L.deinit()
    return out
