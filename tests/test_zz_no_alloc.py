"""The allocation-free entry point g2g_solve_device_noalloc_ against g2g_solve_groups_.

Some callers cannot call cudaMalloc while they run: a host program whose own
allocator has taken all of the GPU's memory, or code that must not allocate in
the middle of its step. For them the library offers one XC build that keeps all
of its intermediates in a fixed device array compiled into the library. This
file checks, through the C ABI, that its energy and Kohn-Sham matrices equal
those of the regular entry point within the parity tolerances, on two calls in
a row (the array keeps the previous call's contents, so the second call would
expose anything that depended on it starting clean), that the calls leave the
device's free memory unchanged, and that it refuses with an error, allocating
nothing, both a grid too large for the array and a grid built in the
tensor-core form (which does not keep the FP64 basis values this path reads).

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C
import os

import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H

pytestmark = pytest.mark.gpu

PROD = os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so")


def _noalloc(L, wl, stream):
    import torch

    npk = wl.basis.M * (wl.basis.M + 1) // 2
    dev = torch.device("cuda")
    if wl.open_shell:
        ra = torch.tensor(wl.rho_a, dtype=torch.float64, device=dev)
        rb = torch.tensor(wl.rho_b, dtype=torch.float64, device=dev)
    else:
        ra = torch.tensor(wl.rho, dtype=torch.float64, device=dev)
        rb = None
    ka = torch.zeros(npk, dtype=torch.float64, device=dev)
    kb = torch.zeros(npk, dtype=torch.float64, device=dev) if wl.open_shell else None
    e = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    vp = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    L.lib.g2g_solve_device_noalloc_.restype = C.c_int
    rc = L.lib.g2g_solve_device_noalloc_(vp(ra), vp(rb), vp(ka), vp(kb), vp(e), C.c_void_p(stream.cuda_stream))
    stream.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    msg = L.check("g2g_solve_device_noalloc_", raise_=False)
    # nothing was allocated on the device during the call (cudaMalloc takes at
    # least one 2 MiB page out of the free memory)
    assert free_after == free_before, (free_before, free_after)
    return rc, msg, float(e.cpu()[0]), ka.cpu().numpy(), (kb.cpu().numpy() if kb is not None else None)


@pytest.mark.parametrize("make", [lambda: W.small_workload(10, 31, 9, True),
                                  lambda: W.make_workload("cfg2-molecule-194", {"C": 16, "N": 4, "O": 4, "H": 40},
                                                          14.0, 2000, 9, False, 194, 40, nocc=62)],
                         ids=["open-pbe-10", "closed-pbe-64-multibatch"])
def test_noalloc_matches_regular_entry_point(make):
    import torch

    wl = make()
    L = H.lib(PROD, True)
    E_ref, K_ref, Kb_ref = H.run(L, wl, precision=0)
    stream = torch.cuda.Stream()
    for call in range(2):
        rc, msg, E, K, Kb = _noalloc(L, wl, stream)
        assert rc == 0 and msg is None, msg
        assert abs(E - E_ref) <= H.E_TOL, (call, E, E_ref)
        assert np.max(np.abs(K - K_ref)) <= H.K_TOL, call
        if wl.open_shell:
            assert np.max(np.abs(Kb - Kb_ref)) <= H.K_TOL, call


def test_noalloc_rejects_grid_beyond_its_array():
    import torch

    # one 60-bohr cube and no spheres: a single group whose intermediates
    # exceed the fixed array
    wl = W.small_workload(20, 5, 9, False)
    L = H.lib(PROD, True)
    H.run(L, wl, precision=0, options=dict(lcs=60.0, sr=0.0))
    rc, msg, E, K, _ = _noalloc(L, wl, torch.cuda.Stream())
    assert rc != 0
    assert msg is not None and "bytes of scratch" in msg
    assert np.isnan(E) and not np.any(K)


def test_noalloc_refuses_tensor_core_grid():
    import torch

    # the default form keeps int8 operands, not the FP64 basis values this
    # entry point reads; building them would allocate, so the call is refused
    wl = W.small_workload(10, 31, 9, True)
    L = H.lib(PROD, True)
    H.run(L, wl, precision=1)
    rc, msg, E, K, Kb = _noalloc(L, wl, torch.cuda.Stream())
    assert rc != 0
    assert msg is not None and "g2g_set_precision_(0)" in msg
    assert np.isnan(E) and not np.any(K) and not np.any(Kb)
    # the regular entry point still works on the same grid afterwards
    E_ref, K_ref, Kb_ref = H.oracle_result(wl)
    E2, K2, Kb2 = H.run(L, wl, precision=1)
    assert abs(E2 - E_ref) <= H.E_TOL
    assert max(np.max(np.abs(K2 - K_ref)), np.max(np.abs(Kb2 - Kb_ref))) <= H.K_TOL
