"""The XC build service on the GPU (include/lio_serve.h).

* Each request's result is the same alone and in the mix: every molecule's
  build is run once by itself, then all builds (several per molecule, with
  different densities) are submitted at once so they overlap on the device; the
  results agree to summation-order noise of the Kohn-Sham atomics.
* The service's result equals the single-molecule C ABI (g2g_solve_groups_) on
  the same molecule and density, and the FP64 form within the parity
  tolerances (tests/helpers.py).
* Admission by HBM footprint: with a budget that holds only some molecules,
  builds still complete correctly while residents are evicted and re-uploaded.
"""
import numpy as np
import pytest

from lio_b200 import serve as S
from lio_b200 import workloads as W

from . import helpers as H

pytestmark = pytest.mark.gpu

MIX_E = 1e-10   # same build alone vs in the mix: only the atomics' summation order differs
MIX_K = 1e-12


def _molecules():
    return [W.small_workload(6, 101, 9, False), W.small_workload(10, 102, 3, False),
            W.small_workload(9, 103, 9, True), W.small_workload(14, 104, 9, False, n_ang=302),
            W.small_workload(4, 105, 2, False)]


def _densities(wl, k):
    rng = np.random.default_rng(1000 + k)
    if wl.open_shell:
        return wl.rho_a + (1e-3 * k) * W.pack_lower(np.eye(wl.basis.M), True), wl.rho_b
    return S.perturbed_density(wl, rng), None


def test_results_are_the_same_alone_and_in_the_mix():
    srv = S.XCServer(precision=1, max_inflight=8)
    wls = _molecules()
    mids = [srv.add(wl) for wl in wls]
    jobs = [(mid, k) for k in range(3) for mid in mids]
    dens = {(mid, k): _densities(srv.mols[mid][0], k) for mid, k in jobs}
    alone = {}
    for mid, k in jobs:
        ra, rb = dens[(mid, k)]
        rid = srv.submit(mid, ra, rb)
        alone[(mid, k)] = srv.wait(rid, mid)
    rids = [(srv.submit(mid, *dens[(mid, k)]), mid, k) for mid, k in jobs]
    mixed = {(mid, k): srv.wait(rid, mid) for rid, mid, k in rids}
    st = srv.stats()
    assert st["peak_inflight"] > 1, st  # the mix did overlap
    for key in jobs:
        (e1, ka1, kb1, _), (e2, ka2, kb2, _) = alone[key], mixed[key]
        assert abs(e1 - e2) <= MIX_E, key
        assert np.max(np.abs(ka1 - ka2)) <= MIX_K, key
        if kb1 is not None:
            assert np.max(np.abs(kb1 - kb2)) <= MIX_K, key
    srv.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_service_matches_the_single_molecule_abi(precision):
    wls = _molecules()[:3]
    srv = S.XCServer(precision=precision)
    for wl in wls:
        mid = srv.add(wl)
        ra, rb = S.densities(wl)
        e, ka, kb, _ = srv.wait(srv.submit(mid, ra, rb), mid)
        L = H.lib(H.os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"), True)
        E_ref, K_ref, Kb_ref = H.run(L, wl, precision=0)
        assert abs(e - E_ref) <= H.E_TOL
        assert np.max(np.abs(ka - K_ref)) <= H.K_TOL
        if wl.open_shell:
            assert np.max(np.abs(kb - Kb_ref)) <= H.K_TOL
    srv.close()


def test_admission_by_footprint_evicts_and_reuploads():
    wls = _molecules()
    probe = S.XCServer(precision=1)
    mids = [probe.add(wl) for wl in wls]
    est = [probe.info(m)["footprint"] for m in mids]  # estimates, used before a first upload
    S.run_all(probe, mids, {m: S.densities(probe.mols[m][0]) for m in mids})  # resident: footprints measured
    fps = [probe.info(m)["footprint"] for m in mids]
    probe.close()
    # every molecule fits alone (estimate and measurement), never all at once
    budget = max(max(est), int(max(fps) + 0.5 * (sum(fps) - max(fps))))
    assert budget < sum(fps), (est, fps)
    srv = S.XCServer(precision=1, budget_bytes=budget, max_inflight=4)
    mids = [srv.add(wl) for wl in wls]
    ref = {}
    for rounds in range(2):
        rids = [(srv.submit(m, *S.densities(srv.mols[m][0])), m) for m in mids]
        for rid, m in rids:
            e, ka, _, _ = srv.wait(rid, m)
            if m in ref:
                assert abs(e - ref[m][0]) <= MIX_E
                assert np.max(np.abs(ka - ref[m][1])) <= MIX_K
            ref[m] = (e, ka)
    st = srv.stats()
    assert st["evictions"] >= 1 and st["uploads"] > len(mids), st
    srv.close()


def test_memory_taken_by_another_user_shrinks_the_budget():
    """After the server sized its budget (90 % of the free HBM), another user of
    the GPU (a torch allocation here) takes most of that memory. Loads that run
    out of device memory shrink the budget and are retried after more eviction,
    so every build still completes and equals the build without the squeeze."""
    import torch

    wls = _molecules()
    probe = S.XCServer(precision=1)
    mids = [probe.add(wl) for wl in wls]
    dens = {m: S.densities(probe.mols[m][0]) for m in mids}
    ref = S.run_all(probe, mids, dens)
    fps = [probe.info(m)["footprint"] for m in mids]
    probe.close()
    srv = S.XCServer(precision=1, max_inflight=4)
    mids2 = [srv.add(wl) for wl in wls]
    free, _ = torch.cuda.mem_get_info()
    room = max(fps) + (sum(fps) - max(fps)) // 3 + (256 << 20)  # all molecules never fit at once
    hog = torch.empty(max(free - room, 0), dtype=torch.uint8, device="cuda")
    try:
        for _ in range(2):
            out = S.run_all(srv, mids2, {m2: dens[m] for m2, m in zip(mids2, mids)})
            for m2, m in zip(mids2, mids):
                assert abs(out[m2][0] - ref[m][0]) <= MIX_E
                assert np.max(np.abs(out[m2][1] - ref[m][1])) <= MIX_K
        st = srv.stats()
        assert st["oom_retries"] >= 1 and st["evictions"] >= 1, st
    finally:
        srv.close()
        del hog
        torch.cuda.empty_cache()


def test_large_molecule_after_smaller_ones_in_the_tensor_core_form():
    """Engines of one process share each kernel and its shared-memory limit: a
    molecule with larger point groups built again after smaller molecules were
    prepared still launches (the limit is only ever raised)."""
    big, small = W.small_workload(30, 111, 9, False), W.small_workload(4, 112, 9, False)
    srv = S.XCServer(precision=1, max_inflight=4)
    try:
        mb = srv.add(big)
        e1, k1, _, _ = srv.wait(srv.submit(mb, big.rho), mb)
        ms = srv.add(small)
        srv.wait(srv.submit(ms, small.rho), ms)
        e2, k2, _, _ = srv.wait(srv.submit(mb, big.rho), mb)
        assert abs(e2 - e1) <= MIX_E and np.max(np.abs(k2 - k1)) <= MIX_K
        E_ref, K_ref, _ = H.oracle_result(big)
        assert abs(e2 - E_ref) <= H.E_TOL and np.max(np.abs(k2 - K_ref)) <= H.K_TOL
    finally:
        srv.close()
