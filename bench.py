"""XC grid-integration throughput (grid points per second of one Kohn-Sham XC build).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the 256-atom open-shell PBE cluster (64 C, 16 N, 16 O, 160 H in a
22 A box, seeded), H 2s1p / C,N,O 3s2p1d contracted Cartesian basis, 40 radial
shells x 302-point Lebedev angular grid per atom, random orthonormal-orbital
alpha/beta densities (N_alpha = N_beta + 2). Synthetic, seeded data; no public
dataset is involved.

A step is one XC build of that molecule: the g2g_solve_groups_(0) work
(density and its derivatives from the packed density matrices, the PBE point
functional, E_xc, and accumulation into the packed Kohn-Sham matrices).
  value : points / (device time per build) with the density already in HBM
          and the Kohn-Sham accumulators left in HBM (g2g_solve_resident_),
          timed with CUDA events on the library's stream;
  e2e   : the same metric through the public C ABI (g2g_solve_groups_) with
          the caller's host arrays: density H2D, Kohn-Sham D2H and the +=
          into the caller's packed vectors inside the timed region.
With --gpus N > 1 (one process per GPU under torchrun) the ranks share the one
molecule: each builds its cost-balanced share of the groups (g2g_set_shard_)
and one NCCL all-reduce of [E_xc, K] per build sums the shares (inside the
timed region); total work is fixed, scaling is strong.

--impl reference times the reference's own CPU g2g path (compiled from its
sources by oracle/Makefile) on the same molecule with all host cores; the
reference supports only its 50/116/194-point angular tables, so it runs the
40 x 194 grid of that molecule (stated in the line).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lio_b200 import workloads as W  # noqa: E402
from lio_b200.g2g import G2GLibrary, angular_tables  # noqa: E402

METRIC = "grid pts/s XC build (FP32-TC vs FP64 plain, |dE|<1e-6 Ha); served p50/p99 ms"
UNIT = "grid points/s"
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libg2g_ref.so")


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def bind(lib: G2GLibrary, wl: W.Workload):
    e, w = angular_tables(wl.n_ang)
    lib.set_options(eai=True)
    if wl.n_ang == 194:
        lib.bind_workload(wl, {2: (e, w)})
        return 2
    lib.bind_workload(wl, {})
    lib.set_angular_grid(3, e, w)
    return 3


def workload(rank: int, name: str = "cfg3") -> W.Workload:
    if name == "cfg2":  # 64-atom closed-shell PBE, 40x302 (small case for profiling)
        return W.config(2)
    if name == "cfg2-open":  # the same 64 atoms, open-shell PBE (small case of the open-shell kernels)
        return W.make_workload("cfg2-open: 64 atoms 16C4N4O40H, 40x302, open PBE",
                               {"C": 16, "N": 4, "O": 4, "H": 40}, 14.0, 2000, 9, True, 302, 40)
    return W.config(3)


def reference_arm(args, rank, world):
    if rank != 0:
        return None
    wl = W.config(3)
    wl.n_ang = 194
    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    if not os.path.exists(REF_LIB):
        return {"impl": "reference", "unavailable": "oracle/_ref/libg2g_ref.so not built (needs the reference sources)"}
    L = G2GLibrary(REF_LIB, product=False)
    L.init()
    gt = bind(L, wl)
    t0 = time.perf_counter()
    L.reload_atom_positions(gt)
    grid_s = time.perf_counter() - t0
    npts = sum(int(L.partition_group(g, ref=True)["meta"][0]) for g in range(L.num_groups(ref=True)))
    for _ in range(args.warmup):
        L.solve_groups(0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        L.solve_groups(0)
    dt = (time.perf_counter() - t0) / args.steps
    value = npts / dt
    sample = (f"full XC build of the 256-atom open-shell PBE molecule on its 40x194 grid ({npts} points; the "
              f"reference has no 302-point table), g2g_solve_groups_(0) with energy, OpenMP on all host cores")
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "cfg3: 256 atoms 64C16N16O160H open-shell PBE, reference grid 40x194",
                       "points": npts, "grid_build_s": grid_s},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


STAGES = ("density_operands", "density", "functional", "ks_operands", "ks")


def stage_times(L, steps: int):
    """Per-stage device ms of the current precision (events between stages; a separate pass)."""
    import torch

    L.g2g_profile_(C.byref(C.c_uint(1)))
    for _ in range(steps):
        L.g2g_solve_resident_()
    torch.cuda.synchronize()
    stage = (C.c_double * 5)()
    nsol = C.c_int(0)
    L.g2g_stage_times_(stage, C.byref(nsol))
    L.g2g_profile_(C.byref(C.c_uint(0)))
    return [stage[i] / max(1, nsol.value) for i in range(5)]


# DRAM traffic of the dominant kernel. A full-size capture of DRAM counters is
# not taken (too large a workload for a multi-pass capture); the 64-atom
# open-shell case (bench.py --workload cfg2-open, 711,684 points, ncu --set full
# on one k_density_tc launch) moved 1.731 GB (1.634 read + 0.097 written)
# against the 1.285 GB its algorithmic-bytes model below gives: 1.35x. A full
# launch's traffic is estimated as that ratio times its own algorithmic bytes
# (the same byte classes grow with the same partition sums).
SMALL_CASE_TRAFFIC_RATIO = 1.731 / 1.2851
# The same for k_fock_tc: on the 64-atom open-shell case (ncu --set full on one
# launch) it moved 0.879 GB (0.872 read + 0.007 written) against the 0.482 GB
# of its model (A slices re-read once per 32-column tile, 27 % of them from L2).
KS_SMALL_CASE_TRAFFIC_RATIO = 0.8786 / 0.4819
FP64_PEAK_NOMINAL = 37.0e12  # FLOP/s, the B200's nominal FP64 rate (no measured figure exists for it)


def partition_sums(lib):
    """Partition statistics, plus the sum over groups of points x shells (simple functions)."""
    st = lib.partition_stats()
    meta = (C.c_int * 8)()
    pns = 0
    for g in range(st["groups"]):
        lib.lib.g2g_partition_group_(C.byref(C.c_int(g)), meta, None, None, None)
        pns += meta[0] * meta[1]
    st["pns"] = pns
    return st


def roofline_model(st, gga: bool, nspin: int, tc: bool, stage_ms, hbm_gbs: float, bf16_tflops: float):
    """Per-stage algorithmic bytes and FLOPs of one XC build and its roofline time
    (the sum over stages of max(FLOPs / peak, bytes / HBM bandwidth), FLOPs as the
    nominal GEMM counts 2 n m^2 per kind and spin against the measured bf16 rate).
    Bytes count what each stage must read and write once."""
    pts, pm, pm2, pns = st["points"], st["pm"], st["pm2"], st["pns"]
    na, nr, nq = (4, 3, 10) if gga else (1, 1, 1)
    b = {}
    f = {}
    # density operands (tensor-core form): the groups' dense density blocks gathered and cut into slices
    b["density_operands"] = 0.0
    # density: the int8 slices of the basis (na kinds x 6 slices per point and function), the radial sums
    # (nr per point and shell) in the tensor-core form; the FP64 basis values (10 or 1 kinds) in the FP64 form;
    # the per-point quantities written per spin and the point coordinates
    b["density"] = (pm * na * 6.0 + pns * nr * 8.0 if tc else pm * (10 if gga else 1) * 8.0) + \
        pts * (nq * 8.0 * nspin + 24.0)
    f["density"] = 2.0 * pm2 * na * nspin
    b["functional"] = pts * (nq * 8.0 * nspin + 8.0 + 8.0 * nspin)
    # Kohn-Sham operands: F read once with the factors (tensor-core form)
    b["ks_operands"] = (pm * 8.0 + pts * 8.0 * nspin) if tc else 0.0
    # Kohn-Sham: F (and its int8 slices in the tensor-core form) and the factors
    b["ks"] = pm * (8.0 + (6.0 if tc else 0.0)) + pts * 8.0 * nspin
    f["ks"] = 2.0 * pm2 * nspin
    bw = hbm_gbs * 1e9
    stages = {}
    total = 0.0
    for i, name in enumerate(STAGES):
        t = max(f.get(name, 0.0) / (bf16_tflops * 1e12), b.get(name, 0.0) / bw)
        stages[name] = {"bytes": b.get(name, 0.0), "flops": f.get(name, 0.0), "roofline_ms": t * 1e3,
                        "measured_ms": stage_ms[i]}
        total += t
    return stages, total * 1e3


def cpu_baseline(wl: W.Workload, builds: int = 5):
    """Reference CPU g2g path on the same molecule (194-point grid): one warm-up,
    then the median of `builds` timed builds."""
    if not os.path.exists(REF_LIB):
        return None
    wl = W.Workload(**{**wl.__dict__, "n_ang": 194})
    cores = os.cpu_count()
    L = G2GLibrary(REF_LIB, product=False)
    L.init()
    gt = bind(L, wl)
    L.reload_atom_positions(gt)
    npts = sum(int(L.partition_group(g, ref=True)["meta"][0]) for g in range(L.num_groups(ref=True)))
    L.solve_groups(0)
    times = []
    for _ in range(builds):
        t0 = time.perf_counter()
        L.solve_groups(0)
        times.append(time.perf_counter() - t0)
    L.deinit()
    dt = statistics.median(times)
    return {"value": npts / dt, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"median of {builds} timed full XC builds (after one warm-up) of the same molecule on the "
                      f"reference's 40x194 grid, {npts} points, {dt:.2f} s each"}


def ours(args, rank, world):
    import torch

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    # a dedicated stream: the legacy default stream (handle 0) would select the
    # library's own stream, which torch's events do not see
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    wl = workload(rank, args.workload)
    lib = G2GLibrary()
    L = lib.lib
    L.g2g_set_stream_(C.c_void_p(stream.cuda_stream))
    lib.check("g2g_set_stream_")
    gt = bind(lib, wl)
    lib.set_precision(args.precision)
    if world > 1:  # this rank's cost-balanced share of the molecule's groups
        L.g2g_set_shard_(C.byref(C.c_int(rank)), C.byref(C.c_int(world)))
        lib.check("g2g_set_shard_")
    t0 = time.perf_counter()
    msg = lib.reload_atom_positions(gt)
    if msg:
        raise RuntimeError(msg)
    grid_s = time.perf_counter() - t0
    st = lib.partition_stats()
    npts = st["points"]  # the whole molecule's points (the partition is built whole on every rank)
    st_main = partition_sums(lib) if rank == 0 else st
    npacked = wl.basis.M * (wl.basis.M + 1) // 2
    nspin = 2 if wl.open_shell else 1
    # the N > 1 exchange: one all-reduce of [E_xc, K_alpha (, K_beta)] per build
    red = torch.zeros(1 + nspin * npacked, dtype=torch.float64, device="cuda") if world > 1 else None

    def reduce_resident():
        L.g2g_copy_resident_results_(C.c_void_p(red.data_ptr() + 8), C.c_void_p(red.data_ptr() + 8 + 8 * npacked)
                                     if nspin == 2 else None, C.c_void_p(red.data_ptr()))
        torch.distributed.all_reduce(red)

    # end-to-end through the public ABI (host arrays, H2D + D2H + += inside; with
    # N > 1 the shares are summed by an all-reduce of the host results)
    host = torch.zeros(1 + nspin * npacked, dtype=torch.float64, pin_memory=True) if world > 1 else None

    def e2e_step():
        E = lib.solve_groups(0)
        if world > 1:
            host[0] = E
            host[1:1 + npacked] = torch.from_numpy(lib.fock)
            if nspin == 2:
                host[1 + npacked:] = torch.from_numpy(lib.fockb)
            dev_t = host.to("cuda", non_blocking=True)
            torch.distributed.all_reduce(dev_t)
            E = float(dev_t[0].cpu())
        return E

    for _ in range(args.warmup):
        e2e_step()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        E = e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    # the bytes the library moved in the last step (only the packed entries the
    # groups touch, when that is at most half of the matrix), plus the exchange
    xh2d, xd2h = C.c_longlong(0), C.c_longlong(0)
    L.g2g_last_transfer_bytes_(C.byref(xh2d), C.byref(xd2h))
    lib.check("g2g_last_transfer_bytes_")
    h2d_b, d2h_b = xh2d.value, xd2h.value
    if world > 1:
        h2d_b += (1 + nspin * npacked) * 8
        d2h_b += 8

    # device-resident throughput
    L.g2g_solve_resident_.restype = C.c_int
    for _ in range(args.warmup):
        launches = L.g2g_solve_resident_()
        if world > 1:
            reduce_resident()
    lib.check("g2g_solve_resident_")
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            L.g2g_solve_resident_()
            if world > 1:
                reduce_resident()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms, e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms, e2e_ms = float(t[0]), float(t[1])
    total_pts = float(npts)

    # per-stage times (separate profiled pass: events between stages)
    stage_ms = stage_times(L, args.steps)

    # the plain FP64 form on the same molecule and device, for the speed-up
    fp64 = None
    if args.precision == 1 and not args.no_fp64:
        lib.set_precision(0)
        for _ in range(args.warmup):
            L.g2g_solve_resident_()
            if world > 1:
                reduce_resident()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            L.g2g_solve_resident_()
            if world > 1:
                reduce_resident()
        e1.record(stream)
        torch.cuda.synchronize()
        fp64_ms = e0.elapsed_time(e1) / args.steps
        if world > 1:
            t = torch.tensor([fp64_ms], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            fp64_ms = float(t[0])
        fp64_stage = stage_times(L, args.steps)
        fp64 = {"value": total_pts / (fp64_ms * 1e-3), "ms_per_step": fp64_ms,
                "stage_ms": dict(zip(STAGES, fp64_stage))}
        lib.set_precision(args.precision)

    # the same molecule on the reference's 40 x 194 grid (its largest table), beside the 302-point headline
    same_grid = None
    if world == 1 and not args.no_same_grid:
        same_grid = same_grid_run(args, lib, wl, stream)

    if rank != 0:
        return None
    hbm, bf16, src = load_peaks()
    gga = wl.iexch > 3
    tc = args.precision == 1
    st = st_main
    stages, roof_ms = roofline_model(st, gga, nspin, tc, stage_ms, hbm, bf16)
    na = 4 if gga else 1
    # dominant kernel: the density contraction (stage 1), one launch per build. In the tensor-core form its
    # binding resource by this model is the int8 tensor work: 21 slice-pair products (pairs s + t <= 5 of
    # six slices per operand) per nominal product, at the int8 dense rate, twice the measured bf16 rate
    t_dens = stage_ms[1] * 1e-3
    dens_bytes = stages["density"]["bytes"]
    if tc:
        int8_ops = 21.0 * stages["density"]["flops"]
        int8_peak = 2.0 * bf16
        t_tensor, t_hbm = int8_ops / (int8_peak * 1e12), dens_bytes / (hbm * 1e9)
        roof = {"bound": "tensor" if t_tensor >= t_hbm else "hbm", "kernel": "k_density_tc",
                "traffic": SMALL_CASE_TRAFFIC_RATIO * dens_bytes}
        if t_tensor >= t_hbm:
            roof.update(achieved=int8_ops / t_dens / 1e12, peak=int8_peak, unit="TOP/s (int8)",
                        frac=int8_ops / t_dens / 1e12 / int8_peak,
                        peak_source=src + " bf16 x 2 (the int8 dense rate of this part)")
        else:
            roof.update(achieved=dens_bytes / t_dens / 1e9, peak=hbm, unit="GB/s",
                        frac=dens_bytes / t_dens / 1e9 / hbm, peak_source=src)
        roof["hbm_frac"] = dens_bytes / t_dens / 1e9 / hbm
        roof["algorithmic_bytes"] = dens_bytes
    else:
        roof = {"bound": "hbm", "kernel": "k_density_fp64", "achieved": dens_bytes / t_dens / 1e9, "peak": hbm,
                "unit": "GB/s", "frac": dens_bytes / t_dens / 1e9 / hbm, "traffic": None, "peak_source": src}
    # the Kohn-Sham contraction: the larger of its byte and int8-work times against its measured time
    ks = stages["ks"]
    t_ks = stage_ms[4] * 1e-3
    ks_roof = {"kernel": "k_fock_tc" if tc else "k_fock_fp64", "bytes": ks["bytes"],
               "hbm_frac": ks["bytes"] / t_ks / 1e9 / hbm if t_ks > 0 else None}
    if tc and t_ks > 0:
        ks_ops = 21.0 * ks["flops"]
        ks_roof["int8_frac"] = ks_ops / t_ks / 1e12 / (2.0 * bf16)
        ks_roof["traffic"] = KS_SMALL_CASE_TRAFFIC_RATIO * ks["bytes"]
    result = {
        "metric": METRIC, "value": total_pts / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f64" if not tc else "i8-split/f64", "data": "synthetic",
        "config": {"workload": wl.name,
                   "points": npts, "groups": st["groups"], "M": wl.basis.M,
                   "precision": "fp64" if not tc else "tensor (int8 Ozaki slices, exact int32, FP64 outside)",
                   "l2": "inputs larger than L2 (%.1f GB read per build by the density contraction)" % (
                       dens_bytes / 1e9),
                   "grid_build_s": round(grid_s, 3), "E_xc": E},
        "e2e": {"value": total_pts / (e2e_ms * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": h2d_b, "d2h_bytes_per_step": d2h_b},
        "gpu_launches": int(launches) * args.steps,
        "stage_ms": dict(zip(STAGES, stage_ms)),
        "roofline": roof,
        "build_roofline": {"roofline_ms": roof_ms, "measured_ms": ms, "frac": roof_ms / ms,
                           "model": "sum over stages of max(nominal GEMM FLOPs / measured bf16 peak, "
                                    "algorithmic bytes / measured HBM bandwidth)",
                           "stages": stages},
        "ks_roofline": ks_roof,
        "clocks": clk.summary(),
    }
    if fp64 is not None:
        fp64_flops = stages["density"]["flops"] + stages["ks"]["flops"]
        fp64["fp64_frac"] = fp64_flops / (fp64["ms_per_step"] * 1e-3) / FP64_PEAK_NOMINAL
        fp64["fp64_peak"] = "%.0f TFLOP/s nominal" % (FP64_PEAK_NOMINAL / 1e12)
        result["fp64_plain"] = fp64
    if same_grid is not None:
        result["same_grid"] = same_grid
    if world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(wl)
    return result


def same_grid_run(args, lib, wl, stream):
    """The GPU arm on the same molecule's 40 x 194 grid (the grid the reference
    arm runs): device-resident and end-to-end points/s through the same ABI."""
    import torch

    wl194 = W.Workload(**{**wl.__dict__, "n_ang": 194})
    L = lib.lib
    gt = bind(lib, wl194)
    msg = lib.reload_atom_positions(gt)
    if msg:
        raise RuntimeError(msg)
    npts = lib.partition_stats()["points"]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        lib.solve_groups(0)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        lib.solve_groups(0)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    for _ in range(args.warmup):
        L.g2g_solve_resident_()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        L.g2g_solve_resident_()
    e1.record(stream)
    torch.cuda.synchronize()
    res_ms = e0.elapsed_time(e1) / args.steps
    return {"grid": "40x194", "points": npts, "value": npts / (res_ms * 1e-3), "ms_per_step": res_ms,
            "e2e": npts / (e2e_ms * 1e-3), "e2e_ms_per_step": e2e_ms}


def forces_mode(args):
    """XC nuclear forces (g2g_solve_groups_ type 2: E_xc and the forces, no
    Kohn-Sham update) of the 256-atom molecule through the public ABI with host
    arrays; the force kernel's own cost is the difference to an energy-only
    build (type 1) of the same form."""
    import torch

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    wl = workload(0, args.workload)
    lib = G2GLibrary()
    L = lib.lib
    L.g2g_set_stream_(C.c_void_p(stream.cuda_stream))
    gt = bind(lib, wl)
    lib.set_precision(args.precision)
    msg = lib.reload_atom_positions(gt)
    if msg:
        raise RuntimeError(msg)
    st = lib.partition_stats()
    npts, nspin = st["points"], 2 if wl.open_shell else 1

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps, out

    L.g2g_last_force_ms_.restype = C.c_double
    kernel_ms = []

    def force_call():
        out = lib.solve_forces(2)
        kernel_ms.append(L.g2g_last_force_ms_())
        return out

    with ClockSampler(0) as clk:
        f_ms, (E, F) = timed(force_call)
    k_ms = float(np.mean(kernel_ms[-args.steps:]))
    xh2d = C.c_longlong(0)
    lib.lib.g2g_last_transfer_bytes_(C.byref(xh2d), None)
    lib.check("g2g_last_transfer_bytes_")
    e_ms, _ = timed(lambda: lib.solve_groups(1))
    tc = args.precision == 1 and wl.iexch > 3
    hbm, _, src = load_peaks()
    if tc:
        # tensor-core force kernel: reads per (point, function) the int8 slices of F
        # (6 bytes) and the three gradient values (24 bytes) once, per spin from L2
        fbytes = st["pm"] * (6.0 + 24.0)
        roof = {"bound": "hbm", "achieved": fbytes / (k_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": fbytes / (k_ms * 1e-3) / 1e9 / hbm, "traffic": None, "kernel": "k_force_tc",
                "peak_source": src}
    else:
        # FP64 force kernel: G = F P per spin (2 n m^2 flops) and the gradient dots (6 n m)
        flops = nspin * (2.0 * st["pm2"] + 6.0 * st["pm"])
        fp64_peak = 148 * 64 * 2 * 1.965e9 / 1e12  # TFLOP/s: 64 FP64 FMA per clock per SM at the max clock
        roof = {"bound": "fp64", "achieved": flops / (k_ms * 1e-3) / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": flops / (k_ms * 1e-3) / 1e12 / fp64_peak, "traffic": None, "kernel": "k_force_fp64",
                "peak_source": "nominal FP64 FMA rate at the max SM clock"}
    res = {"metric": "grid pts/s XC forces (g2g_solve_groups_ type 2)", "value": npts / (f_ms * 1e-3),
           "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": f_ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if args.precision == 0 else "i8-split/f64", "data": "synthetic",
           "mode": "forces",
           "config": {"workload": wl.name, "points": npts, "atoms": wl.mol.natom,
                      "precision_of_build": args.precision, "max_abs_force": float(np.max(np.abs(F))), "E_xc": E},
           "e2e": {"value": npts / (f_ms * 1e-3), "unit": UNIT,
                   "h2d_bytes_per_step": xh2d.value,
                   "d2h_bytes_per_step": 3 * 8 * wl.mol.natom + 8},
           "energy_only_ms": e_ms, "force_kernel_ms": k_ms, "roofline": roof,
           "clocks": clk.summary()}
    if not args.no_cpu_baseline and os.path.exists(REF_LIB):
        wl2 = W.Workload(**{**wl.__dict__, "n_ang": 194})
        R = G2GLibrary(REF_LIB, product=False)
        R.init()
        R.reload_atom_positions(bind(R, wl2))
        n2 = sum(int(R.partition_group(g, ref=True)["meta"][0]) for g in range(R.num_groups(ref=True)))
        R.solve_forces(2)
        t0 = time.perf_counter()
        R.solve_forces(2)
        dt = time.perf_counter() - t0
        R.deinit()
        res["cpu_baseline"] = {"value": n2 / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                               "sample": f"one timed g2g_solve_groups_(2) (after one warm-up) of the same molecule "
                                         f"on the reference's 40x194 grid, {n2} points, {dt:.2f} s"}
    return res


def md_mode(args):
    """MD-like steps of the 256-atom molecule through the public ABI: each step
    displaces every atom by a seeded N(0, 0.01 bohr) in the caller's position
    array, rebuilds the grid (g2g_reload_atom_positions_: partition with the
    Becke weights on the GPU, device upload, tensor-core operands) and computes
    E_xc and the XC forces (g2g_solve_groups_ type 2). Each call returns with
    its work complete, so a step is timed on the host clock around the two
    calls; the first steps (warm-up) grow the reused host and device buffers."""
    import torch

    torch.cuda.set_device(0)
    wl = workload(0, args.workload)
    lib = G2GLibrary()
    gt = bind(lib, wl)
    # the default form (3: tensor core, operands built with the grid) or FP64
    lib.set_precision(3 if args.precision else 0)
    rng = np.random.default_rng(5)
    r = lib._arrays["r"]
    ph = (C.c_double * 3)()
    rows = []
    with ClockSampler(0) as clk:
        for step in range(args.warmup + args.steps):
            if step:
                r += rng.normal(0.0, 0.01, r.shape)
            t0 = time.perf_counter()
            msg = lib.reload_atom_positions(gt)
            if msg:
                raise RuntimeError(msg)
            t1 = time.perf_counter()
            lib.lib.g2g_grid_timings_(ph)
            E, F = lib.solve_forces(2)
            t2 = time.perf_counter()
            if step >= args.warmup:
                rows.append((1e3 * (t1 - t0), ph[0], ph[1], ph[2], 1e3 * (t2 - t1)))
    a = np.array(rows)
    med = np.median(a, axis=0)
    npts = lib.partition_stats()["points"]
    step_ms = float(np.median(a[:, 0] + a[:, 4]))
    return {"metric": "MD steps/s (grid rebuild + XC energy and forces per geometry)", "value": 1e3 / step_ms,
            "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == 0 else "i8-split/f64", "data": "synthetic", "mode": "md",
            "config": {"workload": wl.name, "atoms": wl.mol.natom, "points": npts,
                       "displacement": "N(0, 0.01 bohr) per coordinate per step, seeded"},
            "grid_build_ms": {"median": float(med[0]), "max": float(a[:, 0].max()), "partition": float(med[1]),
                              "upload": float(med[2]), "operands": float(med[3])},
            "forces_call_ms": float(med[4]), "E_xc_last": E,
            "clocks": clk.summary()}


def batch_mode(args):
    """Many-molecule batch through lio_batch_* (include/lio_serve.h): the
    molecules joined per functional class, one kernel launch per stage and
    class, the classes concurrent. value = grid points / wall seconds of one
    build of every molecule with host arrays in and out (density gather, device
    work, Kohn-Sham scatter), so it is also the end-to-end figure; the same
    batch in the plain FP64 form beside it."""
    from lio_b200 import serve as S

    wls = S.batch_molecules(args.batch)
    dens = [S.densities(wl) for wl in wls]

    def run(precision):
        b = S.XCBatch(wls, precision=precision)
        st = b.stats()
        for _ in range(max(1, args.warmup)):
            b.solve(dens)
        dev = 0.0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            _, _, _, ms = b.solve(dens)
            dev += ms
        dt = (time.perf_counter() - t0) / args.steps
        E, Ka, _, _ = b.solve(dens)
        res = [(float(E[i]), Ka[i].copy()) for i in range(len(wls))]
        b.close()
        return st, dt, dev / args.steps, res

    st, dt, dev_ms, res = run(args.batch_precision)
    st0, dt0, dev_ms0, _ = run(0)
    pts = st["points"]
    # every molecule's E_xc and Kohn-Sham matrix against the oracle (the reference's CPU g2g path on the
    # same 194-point grid), serially on the host cores, after the timing
    errs = oracle_errors(list(zip(wls, res))) if not args.no_oracle else None
    nlda = sum(1 for wl in wls if wl.iexch <= 3)
    return {"metric": METRIC, "value": pts / dt, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "i8-split/f64" if args.batch_precision else "f64", "data": "synthetic",
            "mode": "batch",
            "config": {"workload": f"cfg4: {len(wls)} clusters, 3-40 atoms log-uniform (H:C:N:O 10:4:1:1), "
                                   f"30x194 grids, closed shell, {nlda} LDA-VWN / {len(wls) - nlda} PBE",
                       "points": pts, "grid_build_s": round(st["build_s"], 2), "classes": st["classes"],
                       "class_forms": st["forms"], "class_members": st["members"],
                       "batch_precision": args.batch_precision},
            "device_ms_per_step": dev_ms,
            "e2e": {"value": pts / dt, "unit": UNIT, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
            "fp64_plain": {"value": pts / dt0, "ms_per_step": dt0 * 1e3, "device_ms_per_step": dev_ms0},
            "oracle": errs}


def oracle_errors(cases):
    """Per-molecule |dE_xc| and max |dK| of (workload, (E, K, ...)) results against
    the oracle: the reference CPU g2g path for 194-point grids, the C
    restatement for 302-point grids. Returns the worst of each, how many were
    checked and how many met the tolerances (1e-6 Ha, 1e-7)."""
    from tests import helpers as H

    de, dk, ok = [], [], 0
    for wl, r in cases:
        E_ref, K_ref, _ = H.oracle_result(wl)
        de.append(abs(r[0] - E_ref))
        dk.append(float(np.max(np.abs(r[1] - K_ref))))
        ok += int(de[-1] <= H.E_TOL and dk[-1] <= H.K_TOL)
    return {"checked": len(cases), "within_tolerance": ok, "max_abs_dE": max(de) if de else None,
            "max_abs_dK": max(dk) if dk else None,
            "oracle": "reference CPU g2g path (194-point grids) / C restatement (302-point grids)"}


def serve_mode(args):
    """Served stream: Poisson arrivals of XC builds for resident molecules at a
    sweep of rates (fractions of the measured closed-loop capacity); p50/p99
    latency per rate, for the tensor-core and the FP64 form."""
    from lio_b200 import serve as S

    wls = S.served_molecules(args.molecules, max_atoms=args.max_atoms)
    out = {"metric": METRIC, "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "data": "synthetic", "mode": "serve",
           "config": {"workload": f"cfg5: {len(wls)} resident clusters, 4-{args.max_atoms} atoms log-uniform, "
                                  "40x302 grids, closed-shell PBE, P = P0 + 1e-3 S per request",
                      "duration_s_per_rate": args.duration, "max_inflight": args.inflight}}
    rates = None
    for prec in (args.service_precision, 0):
        srv = S.XCServer(precision=prec, max_inflight=args.inflight)
        mids = [srv.add(wl) for wl in wls]
        dens = {m: S.densities(srv.mols[m][0]) for m in mids}
        S.run_all(srv, mids, dens)  # residency and graphs
        srv.reset_stats()
        t0 = time.perf_counter()
        for _ in range(2):
            S.run_all(srv, mids, dens)
        cap = 2 * len(mids) / (time.perf_counter() - t0)  # builds per second, closed loop
        if rates is None:  # offered loads: fractions of the tensor-core form's capacity, for both forms
            rates = [f * cap for f in (0.25, 0.5, 0.75, 0.9)]
        sweep, samples = [], []
        for rate in rates:
            srv.reset_stats()
            lat, sample, failed = S.serve_poisson(srv, mids, rate, args.duration, seed=int(rate) % 1000)
            st = srv.stats()
            row = {"rate_hz": round(rate, 2), "requests": len(lat), "p50_ms": st["p50_ms"],
                   "p99_ms": st["p99_ms"], "points_per_s": st["points"] / max(st["wall_s"], 1e-9),
                   "peak_inflight": st["peak_inflight"], "evictions": st["evictions"],
                   "failed": failed, "oom_retries": st["oom_retries"]}
            if srv.last_errors:
                row["errors"] = sorted(srv.last_errors)[:3]
                srv.last_errors.clear()
            sweep.append(row)
            samples.append(sample)
        forms = [srv.form(m)[0] for m in mids]
        srv.close()
        if prec == args.service_precision and not args.no_oracle:
            # 1 % of the requests were sampled; at most `oracle_spots` of them per rate are checked against the
            # oracle (the C restatement, single-threaded, seconds per molecule on these 302-point grids)
            for row, sample in zip(sweep, samples):
                if sample:
                    picked = sample[:args.oracle_spots]
                    cases = [(W.Workload(**{**wls[mids.index(mid)].__dict__, "rho": rho}), (e, ka))
                             for mid, rho, e, ka in picked]
                    row["oracle_spot_checks"] = oracle_errors(cases)
                    row["sampled_requests"] = len(sample)
        out["tensor" if prec else "fp64_plain"] = {
            "capacity_builds_per_s": cap, "sweep": sweep,
            "forms": {"tensor": sum(1 for f in forms if f == 1), "fp64": sum(1 for f in forms if f == 0)}}
    top = out["tensor"]["sweep"][-1]
    out.update(value=top["points_per_s"], p50_ms=top["p50_ms"], p99_ms=top["p99_ms"],
               dtype="i8-split/f64" if args.service_precision else "f64")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=1, help="1 = tensor-core form (default), 0 = FP64 plain")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 form's comparison timing")
    ap.add_argument("--no-same-grid", action="store_true",
                    help="skip the timing on the molecule's 40x194 grid (the reference arm's grid)")
    ap.add_argument("--mode", default="single", choices=["single", "batch", "serve", "forces", "md"],
                    help="single = the headline 256-atom build; batch = the 512-molecule batch; "
                         "serve = Poisson-arrival serving of 64 resident molecules; "
                         "forces = XC nuclear forces of the 256-atom molecule; "
                         "md = grid rebuild + forces per displaced geometry of the 256-atom molecule")
    ap.add_argument("--batch", type=int, default=512, help="molecules in the batch mode")
    ap.add_argument("--molecules", type=int, default=64, help="resident molecules in the serve mode")
    ap.add_argument("--max-atoms", type=int, default=200, help="largest molecule in the serve mode")
    ap.add_argument("--duration", type=float, default=4.0, help="seconds per arrival rate in the serve mode")
    ap.add_argument("--inflight", type=int, default=32, help="builds on the GPU at once (batch / serve)")
    ap.add_argument("--service-precision", type=int, default=1,
                    help="form of the serve mode: 0 FP64, 1 tensor core (lean: the whole population stays "
                         "resident), 2 autotuned per molecule")
    ap.add_argument("--no-oracle", action="store_true", help="batch / serve: skip the checks against the oracle")
    ap.add_argument("--batch-precision", type=int, default=1,
                    help="batch: 0 FP64, 1 tensor core (classes it cannot run take FP64), 2 autotuned per class")
    ap.add_argument("--oracle-spots", type=int, default=3,
                    help="serve: sampled requests checked against the oracle per arrival rate")
    ap.add_argument("--workload", default="cfg3", choices=["cfg3", "cfg2", "cfg2-open"],
                    help="cfg3 = the 256-atom headline workload; cfg2 / cfg2-open = the 64-atom closed- and "
                         "open-shell cases used for ncu captures")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        res = reference_arm(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if args.mode != "single":
        if rank == 0:
            fn = {"batch": batch_mode, "serve": serve_mode, "forces": forces_mode, "md": md_mode}[args.mode]
            print(json.dumps(fn(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = ours(args, rank, world)
    if res is not None:
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch

        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
