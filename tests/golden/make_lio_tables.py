"""Makes tests/golden/lio_angular_tables.npz: the angular tables lioamber hands
to g2g_parameter_init_ (e_, e_2, e3 and wang, wang2, wang3 for grid types 0, 1
and 2), evaluated from the assignments of lioamber/grid.f90:39-476 as
lioamber computes them in FP64 (pi = 3.14159265358979312D0,
lioamber/liomods/garcha_mod.f:42; sq2 = sqrt(0.5), ssq3 = 1/sqrt(3); the
weights multiplied by 4 pi).

Run from the repository root in a tree that holds the reference:

    python tests/golden/make_lio_tables.py [<reference root>]   (default: beside the repository)

The statements of that subroutine are literal assignments, `do` loops that fill
weight ranges and whole-array scalings; this script evaluates exactly those
forms and fails on anything else.
"""
import math
import os
import re
import sys

import numpy as np

PI = 3.14159265358979312


def parse(src: str):
    body = src[src.index("pi4  = 4.D0 * pi"):src.index("end subroutine gridlio")]
    env = {"pi": PI}
    arrays = {"e_": np.zeros((50, 3)), "e_2": np.zeros((116, 3)), "e3": np.zeros((194, 3)),
              "wang": np.zeros(50), "wang2": np.zeros(116), "wang3": np.zeros(194)}

    def value(expr: str) -> float:
        expr = expr.strip()
        sign = 1.0
        if expr.startswith("-"):
            sign, expr = -1.0, expr[1:].strip()
        elif expr.startswith("+"):
            expr = expr[1:].strip()
        if re.fullmatch(r"[0-9.]+D[+-]?[0-9]+", expr):
            return sign * float(expr.replace("D", "e"))
        if expr in env:
            return sign * env[expr]
        raise ValueError(f"unsupported expression {expr!r}")

    lines = [ln.split("!")[0] for ln in body.splitlines()]
    stmts = []
    for ln in lines:
        stmts += [s.strip() for s in ln.split(";") if s.strip()]
    i = 0
    while i < len(stmts):
        s = stmts[i]
        m = re.fullmatch(r"do icount = (\d+)\s*,\s*(\d+)", s)
        if m:
            lo, hi = int(m.group(1)), int(m.group(2))
            inner = stmts[i + 1]
            assert stmts[i + 2] == "enddo", stmts[i + 2]
            mm = re.fullmatch(r"(wang\d?)\(icount\)\s*=\s*(.+)", inner)
            assert mm, inner
            arrays[mm.group(1)][lo - 1:hi] = value(mm.group(2))
            i += 3
            continue
        if s == "pi4  = 4.D0 * pi":
            env["pi4"] = 4.0 * PI
        elif s == "sq2  = sqrt(0.5000000000000D0)":
            env["sq2"] = math.sqrt(0.5)
        elif s == "ssq3 = 1.D0 / sqrt(3.D0)":
            env["ssq3"] = 1.0 / math.sqrt(3.0)
        elif re.fullmatch(r"(e_|e_2|e3)\s*=\s*0\.0D0", s):
            arrays[s.split("=")[0].strip()][:] = 0.0
        elif re.fullmatch(r"(wang\d?)\s*=\s*\1\s*\*\s*pi4", s):
            name = s.split("=")[0].strip()
            arrays[name] = arrays[name] * env["pi4"]
        else:
            m = re.fullmatch(r"(e_|e_2|e3)\s*\(\s*(\d+)\s*,\s*(\d)\s*\)\s*=\s*(.+)", s)
            if m:
                arrays[m.group(1)][int(m.group(2)) - 1, int(m.group(3)) - 1] = value(m.group(4))
            else:
                m = re.fullmatch(r"([a-z][a-z0-9]*)\s*=\s*(.+)", s)
                if not m:
                    raise ValueError(f"unsupported statement {s!r}")
                env[m.group(1)] = value(m.group(2))
        i += 1
    return arrays


def main(ref_root: str):
    src = open(os.path.join(ref_root, "lioamber", "grid.f90")).read()
    a = parse(src)
    for e, w in (("e_", "wang"), ("e_2", "wang2"), ("e3", "wang3")):
        norms = np.linalg.norm(a[e], axis=1)
        assert np.allclose(norms, 1.0, atol=1e-10), (e, norms.min(), norms.max())
        assert abs(a[w].sum() - 4.0 * PI) < 1e-9, (w, a[w].sum())
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lio_angular_tables.npz")
    np.savez(out, e0=a["e_"], w0=a["wang"], e1=a["e_2"], w1=a["wang2"], e2=a["e3"], w2=a["wang3"])
    print("wrote", out)


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(here, os.pardir, os.pardir, os.pardir, "reference"))
