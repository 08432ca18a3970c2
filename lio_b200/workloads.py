"""Seeded synthetic molecules, bases and density matrices for the XC-build workloads.

Everything here builds the arrays that lioamber's Fortran side hands to
g2g_parameter_init_ (lioamber/drive.f90:176-180 -> g2g/init.cpp:69-81), in the
same conventions:

* coordinates in bohr, converted from angstrom with 0.529177 A/bohr;
* basis order: all s functions, then p (x,y,z consecutive), then d
  (xx,xy,yy,xz,yz,zz), each block in atom order (lioamber/basis_data.f90:1007-1064);
* primitive coefficients carry LIO's primitive normalisation
  (lioamber/basis_data.f90:633-656); `a`/`c` are M x 13 column-major;
* Rm per atomic number = Slater radius / (2 * 0.529177) with the Slater radius a
  Fortran default-REAL literal (lioamber/grid.f90:16-20,33-37), i.e. rounded to
  float32 first;
* packed density matrices are the lower triangle in Fortran 'L' order with the
  off-diagonal elements doubled (lioamber/SCF_aux.f90:31-43).

Workloads (no public dataset is involved; all inputs are seeded synthetic data):
  cfg1  8 atoms (2C,6H), 6 A box, 40x194 grid, closed LDA-VWN, 9 occupied orbitals
  cfg2  64 atoms (16C,4N,4O,40H), 14 A box, 40x302, closed PBE, 62 occupied orbitals
  cfg3  256 atoms (64C,16N,16O,160H), 22 A box, 40x302, open PBE, N_alpha = N_beta + 2
  cfg4  many molecules of 3-40 atoms (H:C:N:O = 10:4:1:1), 30x194, 50% LDA / 50% PBE
  cfg5  resident molecules of 4-200 atoms, 40x302, PBE, P = P0 + eps*S per request
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

BOHR_ANGSTROM = 0.529177
MAX_CONTRACTIONS = 13
Z_OF = {"H": 1, "C": 6, "N": 7, "O": 8}
# (n_s, n_p, n_d) contracted shells per element
SHELLS = {"H": (2, 1, 0), "C": (3, 2, 1), "N": (3, 2, 1), "O": (3, 2, 1)}
AMAX = {"H": 50.0, "C": 5.0e3, "N": 5.0e3, "O": 5.0e3}
EXP_RATIO = 3.0
K_PRIM = 3
# Slater radii (angstrom) of the elements used here, as LIO's table holds them.
SLATER_RADIUS = {1: 0.35, 6: 0.70, 7: 0.65, 8: 0.60}
# LIO's radial shell counts for grid type 0 (lioamber/grid.f90:23-26)
NR_GRID0 = {1: 20, 6: 25, 7: 25, 8: 25}
PI32 = math.pi ** 1.5


@dataclasses.dataclass
class Molecule:
    symbols: list
    Z: np.ndarray        # (natom,) int
    pos: np.ndarray      # (natom, 3) bohr, row-major

    @property
    def natom(self) -> int:
        return len(self.symbols)


@dataclasses.dataclass
class Basis:
    M: int
    nuc: np.ndarray      # (M,) uint32, 1-based atom index
    ncont: np.ndarray    # (M,) uint32
    a: np.ndarray        # (M, 13) float64 (Fortran column-major when passed)
    c: np.ndarray        # (M, 13) float64
    nshell: np.ndarray   # (3,) uint32: s count, p count*3, d count*6
    lmom: np.ndarray     # (M,) angular momentum of each function


@dataclasses.dataclass
class Workload:
    name: str
    mol: Molecule
    basis: Basis
    iexch: int
    open_shell: bool
    n_ang: int
    n_rad: int
    rho: np.ndarray          # packed total density (doubled off-diagonals)
    rho_a: np.ndarray | None
    rho_b: np.ndarray | None
    seed: int
    nco: int = 0
    nunp: int = 0


def random_cluster(counts: dict, box_angstrom: float, seed: int, min_dist: float = 0.9) -> Molecule:
    rng = np.random.default_rng(seed)
    symbols = []
    for sym in ("C", "N", "O", "H"):
        symbols += [sym] * counts.get(sym, 0)
    pos = []
    tries = 0
    while len(pos) < len(symbols):
        p = rng.uniform(0.0, box_angstrom, 3)
        tries += 1
        if tries > 2_000_000:
            raise RuntimeError("could not place atoms without overlap")
        if all(np.linalg.norm(p - q) >= min_dist for q in pos):
            pos.append(p)
    pos = np.array(pos) / BOHR_ANGSTROM
    Z = np.array([Z_OF[s] for s in symbols], dtype=np.int64)
    return Molecule(symbols, Z, pos)


def _prim_norm(a: float, l: int) -> float:
    base = math.sqrt(8.0 * a ** 3)
    if l == 0:
        return math.sqrt(base / PI32)
    if l == 1:
        return math.sqrt(base * 4.0 * a / PI32)
    return math.sqrt(base * 16.0 * a ** 2 / PI32)


def build_basis(mol: Molecule, seed: int) -> Basis:
    """Per element one geometric exponent series amax * 3^-q; s contraction k uses
    q = 3k..3k+2, p and d contractions reuse the most diffuse blocks of the series
    (p: the last n_p blocks, d: the last n_d blocks). Contraction coefficients are
    seeded uniform in [0.2, 1.0] per element and shell, then scaled by LIO's
    primitive normalisation."""
    rng = np.random.default_rng(seed)
    shell_table = {}
    for sym in sorted(set(mol.symbols)):
        ns, npp, nd = SHELLS[sym]
        nq = K_PRIM * ns
        expo = AMAX[sym] / EXP_RATIO ** np.arange(nq)
        shells = []
        for k in range(ns):
            shells.append((0, expo[K_PRIM * k: K_PRIM * (k + 1)]))
        for k in range(npp):
            blk = ns - npp + k
            shells.append((1, expo[K_PRIM * blk: K_PRIM * (blk + 1)]))
        for k in range(nd):
            blk = ns - nd + k
            shells.append((2, expo[K_PRIM * blk: K_PRIM * (blk + 1)]))
        coefs = [rng.uniform(0.2, 1.0, K_PRIM) for _ in shells]
        shell_table[sym] = list(zip(shells, coefs))

    funcs = {0: [], 1: [], 2: []}
    for ia, sym in enumerate(mol.symbols):
        for (l, ex), cf in shell_table[sym]:
            ncomp = (1, 3, 6)[l]
            for _ in range(ncomp):
                funcs[l].append((ia + 1, ex, cf, l))
    allf = funcs[0] + funcs[1] + funcs[2]
    M = len(allf)
    a = np.zeros((M, MAX_CONTRACTIONS))
    c = np.zeros((M, MAX_CONTRACTIONS))
    nuc = np.zeros(M, dtype=np.uint32)
    ncont = np.zeros(M, dtype=np.uint32)
    lmom = np.zeros(M, dtype=np.int64)
    for i, (atom, ex, cf, l) in enumerate(allf):
        nuc[i] = atom
        ncont[i] = len(ex)
        lmom[i] = l
        for k in range(len(ex)):
            a[i, k] = ex[k]
            c[i, k] = _prim_norm(float(ex[k]), l) * cf[k]
    nshell = np.array([len(funcs[0]), len(funcs[1]), len(funcs[2])], dtype=np.uint32)
    return Basis(M, nuc, ncont, a, c, nshell, lmom)


def pack_lower(P: np.ndarray, double_offdiag: bool) -> np.ndarray:
    """Fortran 'L' packed storage: for each column j, rows i >= j (0-based index
    j*M - j(j-1)/2 + (i-j), the packed index of g2g/partition.cpp:64-66)."""
    M = P.shape[0]
    iu = np.triu_indices(M)  # (row r, col c) with r <= c, ordered row-major
    vals = P[iu].copy()
    if double_offdiag:
        vals[iu[0] != iu[1]] *= 2.0
    return vals


def unpack_lower(vec: np.ndarray, M: int) -> np.ndarray:
    out = np.zeros((M, M))
    iu = np.triu_indices(M)
    out[iu] = vec
    out[(iu[1], iu[0])] = vec
    return out


def random_orbitals(M: int, nocc: int, rng) -> np.ndarray:
    C = rng.standard_normal((M, nocc))
    q, _ = np.linalg.qr(C)
    return q


def density_closed(M: int, nocc: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    C = random_orbitals(M, nocc, rng)
    return 2.0 * C @ C.T


def density_open(M: int, nalpha: int, nbeta: int, seed: int):
    rng = np.random.default_rng(seed)
    Ca = random_orbitals(M, nalpha, rng)
    Cb = random_orbitals(M, nbeta, rng)
    return Ca @ Ca.T, Cb @ Cb.T


def make_workload(name: str, counts: dict, box: float, seed: int, iexch: int, open_shell: bool,
                  n_ang: int, n_rad: int, nocc: int | None = None) -> Workload:
    mol = random_cluster(counts, box, seed)
    basis = build_basis(mol, seed + 1)
    M = basis.M
    nelec = int(sum(mol.Z))
    if open_shell:
        nbeta = (nelec - 2) // 2
        nalpha = nbeta + 2
        Pa, Pb = density_open(M, nalpha, nbeta, seed + 2)
        rho_a = pack_lower(Pa, True)
        rho_b = pack_lower(Pb, True)
        rho = rho_a + rho_b
        return Workload(name, mol, basis, iexch, True, n_ang, n_rad, rho, rho_a, rho_b, seed,
                        nco=nbeta, nunp=2)
    nocc = nocc if nocc is not None else nelec // 2
    P = density_closed(M, nocc, seed + 2)
    return Workload(name, mol, basis, iexch, False, n_ang, n_rad, pack_lower(P, True), None, None,
                    seed, nco=nocc)


def config(n: int) -> Workload:
    if n == 1:
        return make_workload("cfg1: 8 atoms 2C6H, 40x194, closed LDA-VWN", {"C": 2, "H": 6}, 6.0,
                             1000, 3, False, 194, 40, nocc=9)
    if n == 2:
        return make_workload("cfg2: 64 atoms 16C4N4O40H, 40x302, closed PBE",
                             {"C": 16, "N": 4, "O": 4, "H": 40}, 14.0, 2000, 9, False, 302, 40, nocc=62)
    if n == 3:
        return make_workload("cfg3: 256 atoms 64C16N16O160H, 40x302, open PBE",
                             {"C": 64, "N": 16, "O": 16, "H": 160}, 22.0, 3000, 9, True, 302, 40)
    raise ValueError(n)


def small_workload(natoms: int, seed: int, iexch: int, open_shell: bool, n_ang: int = 194,
                   n_rad: int = 40, box: float | None = None) -> Workload:
    """A cluster of `natoms` atoms with the H:C:N:O = 10:4:1:1 composition of the
    many-molecule workload; used for parity cases and batches."""
    rng = np.random.default_rng(seed)
    weights = np.array([10, 4, 1, 1], dtype=float)
    syms = rng.choice(["H", "C", "N", "O"], size=natoms, p=weights / weights.sum())
    counts = {s: int(np.sum(syms == s)) for s in ("H", "C", "N", "O")}
    if box is None:
        box = max(3.0, 2.2 * natoms ** (1.0 / 3.0) + 1.5)
    return make_workload(f"cluster{natoms}-seed{seed}", counts, box, seed, iexch, open_shell,
                         n_ang, n_rad)


def rm_table() -> np.ndarray:
    """Rm indexed by atomic number 0..54 as lioamber passes it (entries for the
    elements used here; others are unused placeholders)."""
    rm = np.ones(55)
    for z, r in SLATER_RADIUS.items():
        rm[z] = float(np.float32(r)) / (2.0 * BOHR_ANGSTROM)
    return rm


def shell_tables(n_rad: int):
    nr = np.full(55, 25, dtype=np.uint32)
    for z, v in NR_GRID0.items():
        nr[z] = v
    nr2 = np.full(55, n_rad, dtype=np.uint32)
    return nr, nr2
