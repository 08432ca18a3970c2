"""The XC build service's C ABI (include/lio_serve.h) without a GPU: every
declared entry point is exported, and the admission policy (HBM budget, least
recently used idle residents evicted first, busy ones never) decides as
specified."""
import ctypes as C
import os
import re
import subprocess

from . import helpers as H

PROD = os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so")
HEADER = os.path.join(H.ROOT, "include", "lio_serve.h")


def test_library_exports_every_serving_entry_point():
    names = set(re.findall(r"\b(lio_srv_\w+)\s*\(", open(HEADER).read()))
    assert {"lio_srv_create", "lio_srv_submit", "lio_srv_wait", "lio_srv_stats", "lio_srv_add_molecule"} <= names
    out = subprocess.run(["nm", "-D", "--defined-only", PROD], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    assert not (names - exported), names - exported


def _plan(footprint, busy, last_use, budget, used, need):
    L = C.CDLL(PROD)
    n = len(footprint)
    fp = (C.c_ulonglong * max(n, 1))(*footprint)
    bz = (C.c_int * max(n, 1))(*busy)
    lu = (C.c_ulonglong * max(n, 1))(*last_use)
    ev = (C.c_int * max(n, 1))()
    nev = C.c_int(0)
    ok = L.lio_srv_plan_admission(n, fp, bz, lu, C.c_ulonglong(budget), C.c_ulonglong(used), C.c_ulonglong(need),
                                  ev, C.byref(nev))
    return bool(ok), list(ev)[:nev.value]


def test_admission_fits_without_eviction():
    assert _plan([100, 200], [0, 0], [1, 2], budget=1000, used=300, need=500) == (True, [])


def test_admission_evicts_least_recently_used_idle_first():
    # resident: 0 (lru, idle), 1 (busy), 2 (idle, recent), 3 (idle, older than 2)
    ok, ev = _plan([300, 300, 300, 300], [0, 1, 0, 0], [1, 2, 9, 5], budget=1300, used=1200, need=500)
    assert ok and ev == [0, 3]


def test_admission_never_evicts_busy_molecules():
    ok, ev = _plan([500, 500], [1, 1], [1, 2], budget=1000, used=1000, need=100)
    assert not ok and ev == []


def test_admission_rejects_a_molecule_larger_than_the_budget():
    ok, ev = _plan([], [], [], budget=1000, used=0, need=1001)
    assert not ok and ev == []


def test_non_resident_molecules_are_not_evicted():
    # footprint 0 = not resident
    ok, ev = _plan([0, 400], [0, 0], [1, 2], budget=500, used=400, need=300)
    assert ok and ev == [1]
