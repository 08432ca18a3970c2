"""ctypes binding of the XC build service (include/lio_serve.h) and the two
multi-molecule workloads built on it: a many-molecule batch (all builds
submitted at once) and a served stream (Poisson arrivals, p50/p99 latency).

The service itself is C++ (lio_b200/csrc/serve.cpp): a worker thread owns the
device engines, admits requests by HBM footprint and overlaps the builds of
different molecules on the GPU; Python only describes molecules and submits.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time

import numpy as np

from . import workloads as W
from .g2g import DEFAULT_LIB, angular_tables


class LioMolecule(C.Structure):
    _fields_ = [("natoms", C.c_int), ("xyz", C.POINTER(C.c_double)), ("atomic_number", C.POINTER(C.c_int)),
                ("rm", C.POINTER(C.c_double)), ("shells", C.POINTER(C.c_uint)), ("M", C.c_int),
                ("nuc", C.POINTER(C.c_int)), ("ncont", C.POINTER(C.c_int)), ("a", C.POINTER(C.c_double)),
                ("c", C.POINTER(C.c_double)), ("s_funcs", C.c_int), ("p_funcs", C.c_int), ("d_funcs", C.c_int),
                ("normalize", C.c_int), ("iexch", C.c_int), ("open", C.c_int), ("nang", C.c_int),
                ("ang_x", C.POINTER(C.c_double)), ("ang_y", C.POINTER(C.c_double)),
                ("ang_z", C.POINTER(C.c_double)), ("ang_w", C.POINTER(C.c_double))]


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def molecule_struct(wl: W.Workload):
    """(LioMolecule, keep-alive arrays) for a workload: the same molecule, basis,
    Becke radii, radial shells and angular grid g2g_parameter_init_ receives."""
    mol, bas = wl.mol, wl.basis
    Z = mol.Z.astype(np.int32)
    rm_by_z = W.rm_table()
    _, nr2 = W.shell_tables(wl.n_rad)
    e, w = angular_tables(wl.n_ang)
    keep = dict(
        xyz=np.ascontiguousarray(mol.pos, dtype=np.float64),
        Z=np.ascontiguousarray(Z),
        rm=np.ascontiguousarray(rm_by_z[Z], dtype=np.float64),
        shells=np.ascontiguousarray(nr2[Z], dtype=np.uint32),
        nuc=np.ascontiguousarray(bas.nuc.astype(np.int32) - 1),
        ncont=np.ascontiguousarray(bas.ncont.astype(np.int32)),
        a=np.ascontiguousarray(bas.a, dtype=np.float64),
        c=np.ascontiguousarray(bas.c, dtype=np.float64),
        ex=np.ascontiguousarray(e[:, 0]), ey=np.ascontiguousarray(e[:, 1]), ez=np.ascontiguousarray(e[:, 2]),
        ew=np.ascontiguousarray(w, dtype=np.float64))
    ns = [int(x) for x in bas.nshell]
    s = LioMolecule(mol.natom, _p(keep["xyz"], C.c_double), _p(keep["Z"], C.c_int), _p(keep["rm"], C.c_double),
                    _p(keep["shells"], C.c_uint), bas.M, _p(keep["nuc"], C.c_int), _p(keep["ncont"], C.c_int),
                    _p(keep["a"], C.c_double), _p(keep["c"], C.c_double), ns[0], ns[1] // 3, ns[2] // 6, 1,
                    wl.iexch, 1 if wl.open_shell else 0, len(w), _p(keep["ex"], C.c_double),
                    _p(keep["ey"], C.c_double), _p(keep["ez"], C.c_double), _p(keep["ew"], C.c_double))
    return s, keep


class XCServer:
    """One lio_server: molecules by handle, XC builds by request."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, precision: int = 1, max_inflight: int = 16,
                 path: str = DEFAULT_LIB):
        L = C.CDLL(path)
        L.lio_srv_create.restype = C.c_void_p
        L.lio_srv_create.argtypes = [C.c_int, C.c_ulonglong, C.c_int, C.c_int]
        L.lio_srv_destroy.argtypes = [C.c_void_p]
        L.lio_srv_last_error.restype = C.c_char_p
        L.lio_srv_last_error.argtypes = [C.c_void_p]
        L.lio_srv_add_molecule.argtypes = [C.c_void_p, C.POINTER(LioMolecule)]
        L.lio_srv_molecule_info.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_ulonglong),
                                            C.POINTER(C.c_int)]
        L.lio_srv_submit.restype = C.c_longlong
        L.lio_srv_submit.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.lio_srv_wait.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(C.c_double), C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_double)]
        L.lio_srv_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.lio_srv_molecule_form.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]
        L.lio_srv_reset_stats.argtypes = [C.c_void_p]
        self.L = L
        self.h = L.lio_srv_create(device, budget_bytes, precision, max_inflight)
        self.last_errors = set()
        if not self.h:
            raise RuntimeError("lio_srv_create failed (no CUDA device?)")
        self.mols = {}

    def error(self) -> str:
        return self.L.lio_srv_last_error(self.h).decode(errors="replace")

    def add(self, wl: W.Workload) -> int:
        s, keep = molecule_struct(wl)
        mid = self.L.lio_srv_add_molecule(self.h, C.byref(s))
        if mid < 0:
            raise RuntimeError(self.error())
        self.mols[mid] = (wl, keep)
        return mid

    def info(self, mid: int):
        pts, fp, res = C.c_longlong(0), C.c_ulonglong(0), C.c_int(0)
        if self.L.lio_srv_molecule_info(self.h, mid, C.byref(pts), C.byref(fp), C.byref(res)):
            raise RuntimeError(self.error())
        return dict(points=pts.value, footprint=fp.value, resident=bool(res.value))

    def form(self, mid: int):
        """(form 0 FP64 / 1 tensor core / -1 not uploaded yet, tuned FP64 ms, tuned tensor-core ms)"""
        f, a, b = C.c_int(0), C.c_double(0), C.c_double(0)
        if self.L.lio_srv_molecule_form(self.h, mid, C.byref(f), C.byref(a), C.byref(b)):
            raise RuntimeError(self.error())
        return f.value, a.value, b.value

    def submit(self, mid: int, rho_a: np.ndarray, rho_b: np.ndarray | None = None) -> int:
        ra = np.ascontiguousarray(rho_a, dtype=np.float64)
        rb = None if rho_b is None else np.ascontiguousarray(rho_b, dtype=np.float64)
        rid = self.L.lio_srv_submit(self.h, mid, ra.ctypes.data, None if rb is None else rb.ctypes.data)
        if rid < 0:
            raise RuntimeError(self.error())
        return rid

    def wait(self, rid: int, mid: int):
        wl = self.mols[mid][0]
        npk = wl.basis.M * (wl.basis.M + 1) // 2
        ka = np.zeros(npk)
        kb = np.zeros(npk) if wl.open_shell else None
        e, lat = C.c_double(0), C.c_double(0)
        rc = self.L.lio_srv_wait(self.h, rid, C.byref(e), ka.ctypes.data, None if kb is None else kb.ctypes.data,
                                 C.byref(lat))
        if rc:
            raise RuntimeError(self.error())
        return e.value, ka, kb, lat.value

    def stats(self) -> dict:
        out = (C.c_double * 11)()
        self.L.lio_srv_stats(self.h, out)
        keys = ("completed", "p50_ms", "p99_ms", "mean_ms", "points", "wall_s", "evictions", "uploads",
                "peak_inflight", "oom_retries", "budget")
        return dict(zip(keys, list(out)))

    def reset_stats(self):
        self.L.lio_srv_reset_stats(self.h)

    def close(self):
        if self.h:
            self.L.lio_srv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class XCBatch:
    """One lio_batch: many molecules joined per functional class, each XC build
    stage one kernel launch per class (include/lio_serve.h)."""

    def __init__(self, wls: list, device: int = 0, precision: int = 1, path: str = DEFAULT_LIB):
        L = C.CDLL(path)
        L.lio_batch_create.restype = C.c_void_p
        L.lio_batch_create.argtypes = [C.c_int, C.c_int, C.POINTER(LioMolecule), C.c_int]
        L.lio_batch_create_error.restype = C.c_char_p
        L.lio_batch_last_error.restype = C.c_char_p
        L.lio_batch_last_error.argtypes = [C.c_void_p]
        L.lio_batch_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.lio_batch_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                      C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.lio_batch_destroy.argtypes = [C.c_void_p]
        self.L = L
        self.wls = list(wls)
        structs, self._keep = [], []
        for wl in self.wls:
            st, keep = molecule_struct(wl)
            structs.append(st)
            self._keep.append(keep)
        arr = (LioMolecule * len(structs))(*structs)
        self._arr = arr
        self.h = L.lio_batch_create(device, len(structs), arr, precision)
        if not self.h:
            raise RuntimeError(L.lio_batch_create_error().decode(errors="replace"))
        n = len(self.wls)
        npk = [wl.basis.M * (wl.basis.M + 1) // 2 for wl in self.wls]
        self.fock_a = [np.zeros(k) for k in npk]
        self.fock_b = [np.zeros(k) if wl.open_shell else None for k, wl in zip(npk, self.wls)]
        self.energies = np.zeros(n)
        self._pa = (C.c_void_p * n)(*[f.ctypes.data for f in self.fock_a])
        self._pb = (C.c_void_p * n)(*[(f.ctypes.data if f is not None else None) for f in self.fock_b])

    def stats(self) -> dict:
        pts, ncl, bs = C.c_longlong(0), C.c_int(0), C.c_double(0)
        form, mem = (C.c_int * 16)(), (C.c_int * 16)()
        self.L.lio_batch_stats(self.h, C.byref(pts), C.byref(ncl), C.byref(bs), 16, form, mem)
        return dict(points=pts.value, classes=ncl.value, build_s=bs.value,
                    forms=[form[k] for k in range(min(16, ncl.value))],
                    members=[mem[k] for k in range(min(16, ncl.value))])

    def solve(self, dens: list):
        """dens[i] = (rho_a, rho_b or None): molecule i's packed densities. Returns
        (energies, Kohn-Sham alpha list, beta list, device ms); the Kohn-Sham
        arrays are written (=) and reused by the next call."""
        keep = [(np.ascontiguousarray(a, dtype=np.float64),
                 None if b is None else np.ascontiguousarray(b, dtype=np.float64)) for a, b in dens]
        ra = (C.c_void_p * len(keep))(*[a.ctypes.data for a, _ in keep])
        rb = (C.c_void_p * len(keep))(*[(b.ctypes.data if b is not None else None) for _, b in keep])
        ms = C.c_double(0)
        rc = self.L.lio_batch_solve(self.h, ra, rb, self._pa, self._pb,
                                    self.energies.ctypes.data_as(C.POINTER(C.c_double)), C.byref(ms))
        if rc:
            raise RuntimeError(self.L.lio_batch_last_error(self.h).decode(errors="replace"))
        return self.energies, self.fock_a, self.fock_b, ms.value

    def close(self):
        if self.h:
            self.L.lio_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def densities(wl: W.Workload):
    return (wl.rho_a, wl.rho_b) if wl.open_shell else (wl.rho, None)


# ------------------------------------------------------------- workloads
def batch_molecules(n: int, seed: int = 4000, n_ang: int = 194, n_rad: int = 30):
    """The many-molecule batch: n clusters, atom counts log-uniform over 3-40
    (H:C:N:O = 10:4:1:1), 30 x 194 grids, closed shell, LDA (VWN) and PBE 50/50."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        natoms = int(round(math.exp(rng.uniform(math.log(3), math.log(40)))))
        iexch = 3 if k % 2 == 0 else 9
        out.append(W.small_workload(natoms, seed + k, iexch, False, n_ang=n_ang, n_rad=n_rad))
    return out


def served_molecules(n: int, seed: int = 5000, n_ang: int = 302, n_rad: int = 40, max_atoms: int = 200):
    """The served population: n clusters, atom counts log-uniform over 4-max_atoms, 40 x 302 grids, closed-shell PBE."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        natoms = int(round(math.exp(rng.uniform(math.log(4), math.log(max_atoms)))))
        out.append(W.small_workload(natoms, seed + k, 9, False, n_ang=n_ang, n_rad=n_rad))
    return out


def perturbed_density(wl: W.Workload, rng, eps: float = 1e-3):
    """P = P0 + eps * S (S symmetric with Gaussian entries), packed like P0."""
    M = wl.basis.M
    S = rng.standard_normal((M, M))
    S = 0.5 * (S + S.T)
    return wl.rho + eps * W.pack_lower(S, True)


def serve_poisson(srv: XCServer, mids: list, rate_hz: float, duration_s: float, seed: int = 7,
                  sample_frac: float = 0.01, waiters: int = 32):
    """Poisson arrivals at rate_hz over duration_s, each request for a random
    registered molecule with a fresh perturbed density (P0 + 1e-3 S). Returns the
    per-request latencies (ms, submit to result), for a sample_frac sample
    (molecule, density, E_xc, K) for spot checks against the FP64 form, and the
    number of requests that failed (their errors are not latencies; the distinct
    messages are kept in srv.last_errors)."""
    import queue

    rng = np.random.default_rng(seed)
    lat, sample, failed = [], [], [0]
    lock = threading.Lock()
    todo = queue.Queue()

    def waiter():
        while True:
            item = todo.get()
            if item is None:
                return
            rid, mid, rho, keep = item
            try:
                e, ka, _, ms = srv.wait(rid, mid)
            except RuntimeError as ex:
                with lock:
                    failed[0] += 1
                    srv.last_errors.add(str(ex)[:200])
                continue
            with lock:
                lat.append(ms)
                if keep:
                    sample.append((mid, rho, e, ka))

    pool = [threading.Thread(target=waiter, daemon=True) for _ in range(waiters)]
    for th in pool:
        th.start()
    t_end = time.perf_counter() + duration_s
    t_next = time.perf_counter()
    while True:
        now = time.perf_counter()
        if now >= t_end:
            break
        if now < t_next:
            time.sleep(min(t_next - now, 0.0005))
            continue
        mid = mids[int(rng.integers(len(mids)))]
        rho = perturbed_density(srv.mols[mid][0], rng)
        todo.put((srv.submit(mid, rho), mid, rho, rng.random() < sample_frac))
        t_next += rng.exponential(1.0 / rate_hz)
    for _ in pool:
        todo.put(None)
    for th in pool:
        th.join()
    return lat, sample, failed[0]


def run_all(srv: XCServer, mids: list, dens: dict):
    """Submits one build per molecule at once and waits for all; returns {mid: (E, Ka, Kb)}."""
    rids = [(srv.submit(m, *dens[m]), m) for m in mids]
    out = {}
    for rid, m in rids:
        e, ka, kb, _ = srv.wait(rid, m)
        out[m] = (e, ka, kb)
    return out
