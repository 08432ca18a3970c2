"""ctypes binding of the g2g C ABI (the Fortran-convention entry points lioamber calls).

`G2GLibrary(path)` drives any library that exports that ABI: the B200 library
(lio_b200/libg2g_b200.so) in production, and in the tests also the reference's
own CPU g2g path compiled from its sources. `bind_workload` reproduces what
lioamber's Fortran side passes (lioamber/drive.f90:176-180 ->
g2g/init.cpp:69-81): column-major arrays, 1-based atom indices, caller-owned
density and Fock vectors that must stay alive while the library holds their
pointers.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(HERE, "libg2g_b200.so")

_u = C.c_uint
_pu = C.POINTER(C.c_uint)
_pd = C.POINTER(C.c_double)
_pb = C.POINTER(C.c_bool)


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def angular_tables(n_ang: int):
    """(e column-major n x 3, weights) of the Lebedev grid solved in lebedev.py."""
    data = np.loadtxt(os.path.join(HERE, "data", f"lebedev_{n_ang}.txt"))
    e = np.asfortranarray(data[:, :3])
    return e, np.ascontiguousarray(data[:, 3])


class G2GLibrary:
    def __init__(self, path: str = DEFAULT_LIB, product: bool = True):
        if not os.path.exists(path):
            raise FileNotFoundError(f"g2g library not built: {path} (run python -m lio_b200.build)")
        self.path = path
        self.lib = C.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        self.product = product
        self._keep = []
        L = self.lib
        L.g2g_init_.restype = None
        L.g2g_set_options_.restype = None
        L.g2g_parameter_init_.restype = None
        L.g2g_reload_atom_positions_.restype = None
        L.g2g_new_grid_.restype = None
        L.g2g_solve_groups_.restype = None
        L.g2g_deinit_.restype = None
        if product:
            L.g2g_last_error_.restype = C.c_int
            L.g2g_partition_group_.restype = C.c_int

    # -- reference ABI -------------------------------------------------------
    def init(self):
        self.lib.g2g_init_()

    def set_options(self, fgm=0.0, lcs=8.0, sr=0.6, aaf=False, eai=True, rzw=True, mppc=1, mfe=10,
                    timer=0, verbose=0):
        args = [C.c_double(fgm), C.c_double(lcs), C.c_double(sr), C.c_bool(aaf), C.c_bool(eai),
                C.c_bool(rzw), _u(mppc), _u(mfe), _u(timer), _u(verbose)]
        self._opts = args
        self.lib.g2g_set_options_(*[C.byref(a) for a in args])

    def bind_workload(self, wl: W.Workload, angular: dict | None = None):
        """Calls g2g_parameter_init_ with the arrays lioamber would pass.
        `angular` maps grid type 0/1/2 -> (e, w); missing entries get zero tables."""
        mol, bas = wl.mol, wl.basis
        nat, M = mol.natom, bas.M
        r = np.asfortranarray(mol.pos.astype(np.float64))          # natom x 3, ld = natom
        Rm = W.rm_table()
        Iz = mol.Z.astype(np.uint32)
        Nr, Nr2 = W.shell_tables(wl.n_rad)
        Nuc = bas.nuc.astype(np.uint32).copy()
        ncont = bas.ncont.astype(np.uint32).copy()
        nshell = bas.nshell.astype(np.uint32)
        a = np.asfortranarray(bas.a)
        c = np.asfortranarray(bas.c)
        npacked = M * (M + 1) // 2
        rho = np.ascontiguousarray(wl.rho, dtype=np.float64)
        fock = np.zeros(npacked)
        fockb = np.zeros(npacked)
        if wl.open_shell:
            rhoa = np.ascontiguousarray(wl.rho_a)
            rhob = np.ascontiguousarray(wl.rho_b)
        else:
            rhoa = np.zeros(1)
            rhob = np.zeros(1)
        tables = {}
        for t, n in ((0, 50), (1, 116), (2, 194)):
            if angular and t in angular:
                e, w = angular[t]
            else:
                e, w = np.zeros((n, 3), order="F"), np.zeros(n)
            tables[t] = (np.asfortranarray(e, dtype=np.float64), np.ascontiguousarray(w, dtype=np.float64))
        keep = dict(r=r, Rm=Rm, Iz=Iz, Nr=Nr, Nr2=Nr2, Nuc=Nuc, ncont=ncont, nshell=nshell, a=a, c=c,
                    rho=rho, fock=fock, fockb=fockb, rhoa=rhoa, rhob=rhob, tables=tables)
        self._arrays = keep
        scal = dict(norm=_u(1), natom=_u(nat), max_atoms=_u(nat), ngauss=_u(M), M=_u(M), nco=_u(wl.nco),
                    OPEN=C.c_bool(wl.open_shell), nunp=_u(wl.nunp), nopt=_u(0), iexch=_u(wl.iexch),
                    libxc=C.c_bool(False), ex=_u(0), ec=_u(0))
        self._scal = scal
        self.lib.g2g_parameter_init_(
            C.byref(scal["norm"]), C.byref(scal["natom"]), C.byref(scal["max_atoms"]), C.byref(scal["ngauss"]),
            _ptr(r, C.c_double), _ptr(Rm, C.c_double), _ptr(Iz, C.c_uint), _ptr(Nr, C.c_uint),
            _ptr(Nr2, C.c_uint), _ptr(Nuc, C.c_uint), C.byref(scal["M"]), _ptr(ncont, C.c_uint),
            _ptr(nshell, C.c_uint), _ptr(c, C.c_double), _ptr(a, C.c_double), _ptr(rho, C.c_double),
            _ptr(fock, C.c_double), _ptr(fockb, C.c_double), _ptr(rhoa, C.c_double), _ptr(rhob, C.c_double),
            C.byref(scal["nco"]), C.byref(scal["OPEN"]), C.byref(scal["nunp"]), C.byref(scal["nopt"]),
            C.byref(scal["iexch"]), _ptr(tables[0][0], C.c_double), _ptr(tables[1][0], C.c_double),
            _ptr(tables[2][0], C.c_double), _ptr(tables[0][1], C.c_double), _ptr(tables[1][1], C.c_double),
            _ptr(tables[2][1], C.c_double), C.byref(scal["libxc"]), C.byref(scal["ex"]), C.byref(scal["ec"]))
        self.check("g2g_parameter_init_")

    def set_angular_grid(self, grid_type: int, e: np.ndarray, w: np.ndarray):
        e = np.asfortranarray(e, dtype=np.float64)
        w = np.ascontiguousarray(w, dtype=np.float64)
        self._keep.append((e, w))
        self.lib.g2g_set_angular_grid_(C.byref(_u(grid_type)), C.byref(_u(len(w))), _ptr(e, C.c_double),
                                      _ptr(w, C.c_double))
        self.check("g2g_set_angular_grid_")

    def reload_atom_positions(self, grid_type: int):
        self.lib.g2g_reload_atom_positions_(C.byref(_u(grid_type)))
        return self.check("g2g_reload_atom_positions_", raise_=False)

    def new_grid(self, grid_type: int):
        self.lib.g2g_new_grid_(C.byref(_u(grid_type)))
        return self.check("g2g_new_grid_", raise_=False)

    def solve_groups(self, computation_type: int = 0) -> float:
        e = C.c_double(0.0)
        forces = np.zeros(3 * max(1, self._scal["natom"].value))
        self.lib.g2g_solve_groups_(C.byref(_u(computation_type)), C.byref(e), _ptr(forces, C.c_double))
        self.check("g2g_solve_groups_")
        return e.value

    def solve_forces(self, computation_type: int = 2):
        """g2g_solve_groups_ type 2 (energy + forces) or 3 (forces only): returns
        (E_xc, forces) with forces natoms x 3, the XC gradient contributions the
        library added into a zeroed caller array (column-major, leading
        dimension max_atoms = natoms)."""
        if computation_type not in (2, 3):
            raise ValueError("forces are computation types 2 and 3")
        e = C.c_double(0.0)
        nat = max(1, self._scal["natom"].value)
        forces = np.zeros(3 * nat)
        self.lib.g2g_solve_groups_(C.byref(_u(computation_type)), C.byref(e), _ptr(forces, C.c_double))
        self.check("g2g_solve_groups_")
        return e.value, forces.reshape(3, nat).T.copy()

    def deinit(self):
        self.lib.g2g_deinit_()

    # -- caller-side arrays ---------------------------------------------------
    @property
    def fock(self) -> np.ndarray:
        return self._arrays["fock"]

    @property
    def fockb(self) -> np.ndarray:
        return self._arrays["fockb"]

    def set_density(self, rho=None, rho_a=None, rho_b=None):
        """Overwrites the caller-owned packed density in place (as SCF.f90 does)."""
        if rho is not None:
            self._arrays["rho"][:] = rho
        if rho_a is not None:
            self._arrays["rhoa"][:] = rho_a
        if rho_b is not None:
            self._arrays["rhob"][:] = rho_b

    # -- additions -------------------------------------------------------------
    def check(self, where: str, raise_: bool = True):
        if not self.product:
            return None
        buf = C.create_string_buffer(512)
        code = self.lib.g2g_last_error_(buf, C.byref(_u(512)))
        if code != 0:
            msg = f"{where}: {buf.value.decode(errors='replace')}"
            if raise_:
                raise RuntimeError(msg)
            return msg
        return None

    def set_precision(self, mode: int):
        self.lib.g2g_set_precision_(C.byref(_u(mode)))

    def set_lean(self, on: bool):
        """Lean tensor-core form: the blocked FP64 basis released once the operands are built."""
        self.lib.g2g_set_lean_(C.byref(_u(1 if on else 0)))
        self.check("g2g_set_lean_")

    def set_device_weights(self, on: bool):
        """Becke weights of the next grid builds on the GPU (default) or the host."""
        self.lib.g2g_set_device_weights_(C.byref(_u(1 if on else 0)))
        self.check("g2g_set_device_weights_")

    def partition_stats(self) -> dict:
        out = (C.c_longlong * 6)()
        self.lib.g2g_partition_stats_(out)
        return dict(groups=out[0], cubes=out[1], spheres=out[2], points=out[3], pm=out[4], pm2=out[5])

    def partition_group(self, g: int, ref: bool = False):
        """Group g as a dict (works on the product and, through the accessors of
        the oracle build, on the reference)."""
        meta = (C.c_int * 8)()
        if ref:
            rc = self.lib.ref_group_meta(C.c_int(g), meta)
        else:
            rc = self.lib.g2g_partition_group_(C.byref(C.c_int(g)), meta, None, None, None)
        if rc != 0:
            raise IndexError(g)
        n, nf = meta[0], meta[1]
        ids = np.zeros((n, 3), dtype=np.int32)
        xyzw = np.zeros((n, 4))
        funcs = np.zeros(nf, dtype=np.int32)
        if ref:
            nucs = np.zeros(meta[6], dtype=np.int32)
            self.lib.ref_group_points(C.c_int(g), _ptr(ids, C.c_int), _ptr(xyzw, C.c_double))
            self.lib.ref_group_lists(C.c_int(g), _ptr(funcs, C.c_int), _ptr(nucs, C.c_int))
        else:
            self.lib.g2g_partition_group_(C.byref(C.c_int(g)), meta, _ptr(ids, C.c_int), _ptr(xyzw, C.c_double),
                                          _ptr(funcs, C.c_int))
        return dict(meta=list(meta), ids=ids, xyzw=xyzw, funcs=funcs)

    def num_groups(self, ref: bool = False) -> int:
        if ref:
            return self.lib.ref_num_cubes() + self.lib.ref_num_spheres()
        return self.partition_stats()["groups"]

    def last_timings(self):
        a, b = C.c_double(0), C.c_double(0)
        self.lib.g2g_last_timings_(C.byref(a), C.byref(b))
        return a.value, b.value
