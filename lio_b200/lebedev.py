"""Lebedev angular quadratures on the unit sphere, derived here from first principles.

LIO hard-codes 50/116/194-point angular tables (lioamber/grid.f90:39-476) and the
g2g C ABI receives them as column-major (n x 3) direction arrays plus weights
scaled to 4*pi (g2g/init.cpp:163-174). The 302-point grid (exact to degree 29)
that the 64- and 256-atom workloads use does not exist in the reference, so it
is generated here.

Method: a Lebedev grid is a union of octahedral-group orbits
  a1 (+-1,0,0)         6 points
  a2 (0,+-h,+-h)      12 points, h = 1/sqrt(2)
  a3 (+-t,+-t,+-t)     8 points, t = 1/sqrt(3)
  b  (+-l,+-l,+-m)    24 points, m = sqrt(1-2l^2)
  c  (+-p,+-q,0)      24 points, q = sqrt(1-p^2)
  d  (+-r,+-s,+-u)    48 points, u = sqrt(1-r^2-s^2)
with one weight per orbit. Exactness to degree L for octahedrally invariant
polynomials reduces (odd degrees vanish by symmetry, and on the sphere the
monomials of degree exactly L span all lower even degrees) to the moment
equations  sum_orbit w * sum_pts x^a y^b z^c = I(a,b,c)  for even a>=b>=c,
a+b+c = L. Those are solved by damped least squares from seeded starts and
then polished by Newton iterations; the result is checked against the exact
sphere integrals of every even monomial up to degree L.
"""
from __future__ import annotations

import functools
import itertools
import math

import numpy as np

# orbit structure (number of b, c, d orbits and whether a1/a2/a3 are present)
_STRUCTURE = {
    194: dict(a1=True, a2=True, a3=True, nb=4, nc=1, nd=1, degree=23),
    302: dict(a1=True, a2=False, a3=True, nb=6, nc=2, nd=2, degree=29),
}


def _sphere_moment(a: int, b: int, c: int) -> float:
    """Exact integral of x^a y^b z^c over the unit sphere divided by 4*pi (a,b,c even)."""
    lg = math.lgamma
    v = math.log(2.0) + lg((a + 1) / 2) + lg((b + 1) / 2) + lg((c + 1) / 2) - lg((a + b + c + 3) / 2)
    return math.exp(v) / (4.0 * math.pi)


def _even_monomials(degree: int, exact_only: bool):
    out = []
    degs = [degree] if exact_only else range(0, degree + 1, 2)
    for n in degs:
        for a in range(n, -1, -2):
            for b in range(min(a, n - a), -1, -2):
                c = n - a - b
                if c < 0 or c > b or c % 2:
                    continue
                out.append((a, b, c))
    return out


def _orbit_array(kind, p):
    """Exact (unrounded) points of one orbit as an (k,3) array."""
    if kind == "a1":
        v = (1.0, 0.0, 0.0)
    elif kind == "a2":
        h = math.sqrt(0.5)
        v = (0.0, h, h)
    elif kind == "a3":
        t = 1.0 / math.sqrt(3.0)
        v = (t, t, t)
    elif kind == "b":
        l = p[0]
        v = (l, l, math.sqrt(max(0.0, 1.0 - 2 * l * l)))
    elif kind == "c":
        q = p[0]
        v = (q, math.sqrt(max(0.0, 1.0 - q * q)), 0.0)
    else:
        r, t = p
        v = (r, t, math.sqrt(max(0.0, 1.0 - r * r - t * t)))
    seen = {}
    for perm in itertools.permutations(range(3)):
        for signs in itertools.product((1.0, -1.0), repeat=3):
            pt = tuple(signs[i] * v[perm[i]] for i in range(3))
            key = tuple(round(x, 12) + 0.0 for x in pt)
            if key not in seen:
                seen[key] = pt
    return np.array(sorted(seen.values(), key=lambda t: tuple(round(x, 12) for x in t))[::-1])


def _base_vector(kind, p):
    if kind == "a1":
        return (1.0, 0.0, 0.0)
    if kind == "a2":
        h = math.sqrt(0.5)
        return (0.0, h, h)
    if kind == "a3":
        t = 1.0 / math.sqrt(3.0)
        return (t, t, t)
    if kind == "b":
        l = p[0]
        return (l, l, math.sqrt(max(0.0, 1.0 - 2 * l * l)))
    if kind == "c":
        q = p[0]
        return (q, math.sqrt(max(0.0, 1.0 - q * q)), 0.0)
    r, t = p
    return (r, t, math.sqrt(max(0.0, 1.0 - r * r - t * t)))


def _orbit_sums(kind, p, mons):
    """Sum of x^a y^b z^c over one orbit, for even exponents: sign flips leave each
    term unchanged, so it is 2^(nonzero components) times the sum over the distinct
    permutations of the base vector."""
    v = _base_vector(kind, p)
    nz = sum(1 for t in v if t != 0.0)
    perms = set(itertools.permutations(v))
    E = np.asarray(mons, dtype=float)
    acc = np.zeros(len(mons))
    for pv in perms:
        acc += np.prod(np.power(np.asarray(pv)[None, :], E), axis=1)
    return (2.0 ** nz) * acc


def _unpack(params, st):
    i = 0
    orbits = []
    for k in ("a1", "a2", "a3"):
        if st[k]:
            orbits.append((k, (), params[i]))
            i += 1
    for _ in range(st["nb"]):
        orbits.append(("b", (params[i],), params[i + 1]))
        i += 2
    for _ in range(st["nc"]):
        orbits.append(("c", (params[i],), params[i + 1]))
        i += 2
    for _ in range(st["nd"]):
        orbits.append(("d", (params[i], params[i + 1]), params[i + 2]))
        i += 3
    return orbits


def _residual(params, st, mons, target):
    acc = np.zeros(len(mons))
    for kind, p, w in _unpack(params, st):
        acc += w * _orbit_sums(kind, p, mons)
    return acc / target - 1.0


def _valid(orbits, st) -> bool:
    lb = sorted(p[0] for k, p, w in orbits if k == "b")
    lc = sorted(p[0] for k, p, w in orbits if k == "c")
    if any(w <= 0 for k, p, w in orbits):
        return False
    if any(not (1e-3 < l < math.sqrt(0.5) - 1e-3) or abs(l - 1 / math.sqrt(3)) < 1e-3 for l in lb):
        return False
    if any(b - a < 1e-4 for a, b in zip(lb, lb[1:])):
        return False
    if any(not (1e-3 < q < math.sqrt(0.5) - 1e-3) for q in lc):
        return False
    if any(b - a < 1e-4 for a, b in zip(lc, lc[1:])):
        return False
    for k, p, w in orbits:
        if k == "d":
            r, t = p
            u2 = 1 - r * r - t * t
            if u2 <= 1e-6:
                return False
            u = math.sqrt(u2)
            if not (r > t + 1e-3 and t > u + 1e-3):  # canonical ordering r > s > u > 0
                return False
    dd = sorted(p for k, p, w in orbits if k == "d")
    if any(abs(a[0] - b[0]) + abs(a[1] - b[1]) < 1e-4 for a, b in zip(dd, dd[1:])):
        return False
    return True


def _canonical_d(r, t):
    u = math.sqrt(max(0.0, 1 - r * r - t * t))
    v = sorted((abs(r), abs(t), u), reverse=True)
    return v[0], v[1]


@functools.lru_cache(maxsize=None)
def _solve(npts: int):
    from scipy.optimize import least_squares

    st = _STRUCTURE[npts]
    deg = st["degree"] - 1  # highest even degree
    mons = _even_monomials(deg, exact_only=False)
    target = np.array([_sphere_moment(*m) for m in mons])
    rng = np.random.default_rng(npts)
    nparam = int(st["a1"]) + int(st["a2"]) + int(st["a3"]) + 2 * st["nb"] + 2 * st["nc"] + 3 * st["nd"]
    best = None
    for attempt in range(4000):
        x0 = []
        w0 = 1.0 / npts
        for k in ("a1", "a2", "a3"):
            if st[k]:
                x0.append(w0 * rng.uniform(0.5, 1.5))
        ls = np.sort(rng.uniform(0.05, 0.69, st["nb"]))
        for l in ls:
            x0 += [l, w0 * rng.uniform(0.7, 1.3)]
        for q in np.sort(rng.uniform(0.1, 0.69, st["nc"])):
            x0 += [q, w0 * rng.uniform(0.7, 1.3)]
        for _ in range(st["nd"]):
            while True:
                v = np.abs(rng.normal(size=3))
                v /= np.linalg.norm(v)
                v = np.sort(v)[::-1]
                if v[0] - v[1] > 0.02 and v[1] - v[2] > 0.02 and v[2] > 0.05:
                    break
            x0 += [v[0], v[1], w0 * rng.uniform(0.7, 1.3)]
        x0 = np.array(x0)
        try:
            sol = least_squares(_residual, x0, args=(st, mons, target), xtol=1e-15, ftol=1e-15,
                                gtol=1e-15, max_nfev=4000, method="lm")
        except Exception:
            continue
        res = np.max(np.abs(sol.fun))
        orbits = _unpack(sol.x, st)
        # bring d orbits to canonical form before validation
        orbits = [(k, _canonical_d(*p) if k == "d" else p, w) for k, p, w in orbits]
        if res < 1e-12 and _valid(orbits, st):
            best = orbits
            break
    if best is None:
        raise RuntimeError(f"Lebedev {npts}: moment equations did not converge")
    # Newton polish (square or over-determined, consistent): a few Gauss-Newton steps
    params = []
    for k, p, w in best:
        params += list(p) + [w]
    # params in _unpack order: for orbit kinds the parameter layout is (p..., w) except a* (w)
    x = np.array(params)
    x = _reorder_for_unpack(best, st)
    for _ in range(6):
        f = _residual(x, st, mons, target)
        J = np.empty((len(f), len(x)))
        for j in range(len(x)):
            h = 1e-7 * max(1.0, abs(x[j]))
            xp = x.copy(); xp[j] += h
            xm = x.copy(); xm[j] -= h
            J[:, j] = (_residual(xp, st, mons, target) - _residual(xm, st, mons, target)) / (2 * h)
        dx = np.linalg.lstsq(J, -f, rcond=None)[0]
        x = x + dx
    orbits = _unpack(x, st)
    pts, wts = [], []
    for kind, p, w in orbits:
        arr = _orbit_array(kind, p)
        pts.append(arr)
        wts.append(np.full(len(arr), w))
    pts = np.concatenate(pts)
    wts = np.concatenate(wts)
    assert pts.shape[0] == npts, pts.shape
    return pts, wts


def _reorder_for_unpack(orbits, st):
    x = []
    for k, p, w in orbits:
        if k in ("a1", "a2", "a3"):
            x.append(w)
        else:
            x += list(p) + [w]
    return np.array(x)


def lebedev(npts: int):
    """Return (directions (npts,3) float64, weights (npts,) float64 summing to 4*pi)."""
    pts, wts = _solve(npts)
    return pts.copy(), wts * (4.0 * math.pi)


def max_moment_error(pts: np.ndarray, wts: np.ndarray, degree: int) -> float:
    """Largest |quadrature - exact| / exact over even monomials up to `degree` (weights sum 4*pi)."""
    worst = 0.0
    for (a, b, c) in _even_monomials(degree - (degree % 2), exact_only=False):
        for perm in set(itertools.permutations((a, b, c))):
            q = np.sum(wts * pts[:, 0] ** perm[0] * pts[:, 1] ** perm[1] * pts[:, 2] ** perm[2]) / (4 * math.pi)
            ex = _sphere_moment(*perm)
            worst = max(worst, abs(q - ex) / ex)
    return worst
