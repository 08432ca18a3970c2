"""Multi-GPU sharding of one molecule's groups, without a GPU.

The product assigns the partition's groups to ranks (g2g_shard_groups_:
longest processing time first on the reference's group cost); each rank builds
its groups' share of E_xc and of the Kohn-Sham matrix and one all-reduce sums
them. Here two `gloo` ranks on CPU each take their share from the product's
assignment, build it with the C restatement (the oracle) and all-reduce; the
sums must equal the whole build, every group must have exactly one owner, and
the shares must be balanced."""
import ctypes as C
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from lio_b200 import workloads as W

from . import helpers as H

PROD = os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so")


def _owners(wl, world):
    L = H.lib(PROD, True)
    gt = H.bind(L, wl)
    L.reload_atom_positions(gt)  # without a GPU: reports the missing device after building the partition
    ng = L.num_groups()
    owner = (C.c_int * ng)()
    n = L.lib.g2g_shard_groups_(C.byref(C.c_int(world)), owner)
    assert n == ng
    costs = []
    for g in range(ng):
        meta = L.partition_group(g)["meta"]
        npts, m = meta[0], meta[5]
        costs.append(10 * ((npts * m * (1 + m)) // 2) + 250000)
    return list(owner), costs


def _rank(rank, world, port, wl_args, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    wl = W.small_workload(*wl_args)
    owner, _ = _owners(wl, world)
    mine = [g for g, r in enumerate(owner) if r == rank]
    E, K, Kb, _ = H.restatement(wl, groups=mine)
    t = torch.tensor(np.concatenate([[E], K, Kb]), dtype=torch.float64)
    dist.all_reduce(t)
    if rank == 0:
        np.save(out, t.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("wl_args", [(12, 21, 9, False), (10, 31, 9, True)], ids=["closed-pbe", "open-pbe"])
def test_two_rank_shards_sum_to_the_whole_build(tmp_path, wl_args):
    world, out = 2, str(tmp_path / "sum.npy")
    port = 29500 + (os.getpid() % 2000)
    mp.start_processes(_rank, args=(world, port, wl_args, out), nprocs=world, join=True, start_method="spawn")
    tot = np.load(out)
    wl = W.small_workload(*wl_args)
    E, K, Kb, _ = H.restatement(wl)
    npk = len(K)
    assert abs(tot[0] - E) <= 1e-12
    assert np.max(np.abs(tot[1:1 + npk] - K)) <= 1e-12
    assert np.max(np.abs(tot[1 + npk:] - Kb)) <= 1e-12


def test_assignment_covers_every_group_once_and_balances():
    wl = W.config(2)
    for world in (2, 4, 8):
        owner, costs = _owners(wl, world)
        assert set(owner) == set(range(world))
        load = np.zeros(world)
        for g, r in enumerate(owner):
            load[r] += costs[g]
        # LPT bound: max load <= mean + the largest single group
        assert load.max() <= load.mean() + max(costs) + 1e-9
        assert load.max() / load.mean() < 1.25
