"""Sharded builds on one GPU: the shares of g2g_set_shard_(rank, world) built one
after another in one process add up to the whole build (E_xc and the
Kohn-Sham matrices), in both forms."""
import ctypes as C
import os

import numpy as np
import pytest

from lio_b200 import workloads as W

from . import helpers as H

pytestmark = pytest.mark.gpu

PROD = os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so")


def _share(L, wl, rank, world, precision):
    L.lib.g2g_set_shard_(C.byref(C.c_int(rank)), C.byref(C.c_int(world)))
    try:
        return H.run(L, wl, precision=precision)
    finally:
        L.lib.g2g_set_shard_(C.byref(C.c_int(0)), C.byref(C.c_int(1)))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("world", [2, 3])
def test_shards_add_up_to_the_whole_build(precision, world):
    wl = W.small_workload(14, 77, 9, True, n_ang=302)
    L = H.lib(PROD, True)
    E, K, Kb = _share(L, wl, 0, 1, precision)
    Es, Ks, Kbs = 0.0, np.zeros_like(K), np.zeros_like(Kb)
    for r in range(world):
        e, k, kb = _share(L, wl, r, world, precision)
        Es += e
        Ks += k
        Kbs += kb
    assert abs(Es - E) <= 1e-10
    assert np.max(np.abs(Ks - K)) <= 1e-12
    assert np.max(np.abs(Kbs - Kb)) <= 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_shards_accumulate_into_one_set_of_buffers(precision):
    """g2g_set_accumulators_: every shard's resident solve adds its Kohn-Sham
    contributions (the contraction's own atomics) and E_xc into the same device
    buffers, as the shards of a multi-GPU build add into one GPU's buffers over
    NVLink; the buffers then hold the whole build without any reduction step."""
    import torch

    wl = W.small_workload(14, 77, 9, True, n_ang=302)
    L = H.lib(PROD, True)
    E, K, Kb = _share(L, wl, 0, 1, precision)
    npk = K.size
    acc = torch.zeros(2 * npk + 1, dtype=torch.float64, device="cuda")
    pa, pb, pe = (C.c_void_p(acc.data_ptr() + 8 * o) for o in (0, npk, 2 * npk))
    L.lib.g2g_solve_resident_.restype = C.c_int
    world = 3
    for r in range(world):
        L.lib.g2g_set_shard_(C.byref(C.c_int(r)), C.byref(C.c_int(world)))
        try:
            gt = H.bind(L, wl)
            L.set_precision(precision)
            assert not L.reload_atom_positions(gt)
            L.solve_groups(0)  # uploads the densities; resident solves reuse them
            L.lib.g2g_set_accumulators_(pa, pb, pe)
            L.check("g2g_set_accumulators_")
            for _ in range(2 if r == 0 else 1):  # the first shard twice: graph capture, then replay
                if r == 0:
                    acc.zero_()
                torch.cuda.synchronize()  # the library's stream is not torch's
                assert L.lib.g2g_solve_resident_() > 0
                L.check("g2g_solve_resident_")
                torch.cuda.synchronize()
        finally:
            L.lib.g2g_set_accumulators_(None, None, None)
            L.lib.g2g_set_shard_(C.byref(C.c_int(0)), C.byref(C.c_int(1)))
    torch.cuda.synchronize()
    out = acc.cpu().numpy()
    assert abs(out[2 * npk] - E) <= 1e-10
    assert np.max(np.abs(out[:npk] - K)) <= 1e-12
    assert np.max(np.abs(out[npk:2 * npk] - Kb)) <= 1e-12


def _ipc_shard(rank, world, precision, acc, npk):
    """Child process: build shard `rank` and add it into the parent's buffers,
    which torch maps into this process through CUDA IPC."""
    import torch

    from lio_b200.g2g import G2GLibrary

    wl = W.small_workload(14, 77, 9, True, n_ang=302)
    L = G2GLibrary(PROD)
    L.lib.g2g_set_shard_(C.byref(C.c_int(rank)), C.byref(C.c_int(world)))
    gt = H.bind(L, wl)
    L.set_precision(precision)
    assert not L.reload_atom_positions(gt)
    L.solve_groups(0)  # uploads the densities
    pa, pb, pe = (C.c_void_p(acc.data_ptr() + 8 * o) for o in (0, npk, 2 * npk))
    L.lib.g2g_set_accumulators_(pa, pb, pe)
    L.check("g2g_set_accumulators_")
    L.lib.g2g_solve_resident_.restype = C.c_int
    assert L.lib.g2g_solve_resident_() > 0
    L.check("g2g_solve_resident_")
    torch.cuda.synchronize()
    L.lib.g2g_set_accumulators_(None, None, None)
    L.deinit()


@pytest.mark.parametrize("precision", [0, 1])
def test_shards_in_two_processes_accumulate_through_cuda_ipc(precision):
    """The multi-process form of the fused reduction: two processes (one per
    shard, here on one GPU) add into buffers that a third process owns and
    shares through CUDA IPC, the mapping a multi-GPU build uses over NVLink.
    No kernel waits on another process's kernels."""
    import torch
    import torch.multiprocessing as mp

    wl = W.small_workload(14, 77, 9, True, n_ang=302)
    L = H.lib(PROD, True)
    E, K, Kb = _share(L, wl, 0, 1, precision)
    npk = K.size
    acc = torch.zeros(2 * npk + 1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_ipc_shard, args=(r, 2, precision, acc, npk)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    torch.cuda.synchronize()
    out = acc.cpu().numpy()
    assert abs(out[2 * npk] - E) <= 1e-10
    assert np.max(np.abs(out[:npk] - K)) <= 1e-12
    assert np.max(np.abs(out[npk:2 * npk] - Kb)) <= 1e-12
