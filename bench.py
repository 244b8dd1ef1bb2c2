#!/usr/bin/env python
"""Benchmark: SPECT system-matrix throughput (matrix elements/s) on B200.

Workload (default): the production photoelectric system of configuration 2 — 96x96x32
voxels of 1 mm, a 20 mm tungsten plate with 48x48 hexagonal holes (1.5 mm, pitch 2 mm),
64x64 NaI crystals of 1.6x1.6x6 mm — with the reference's own integration constants
(8x16x8 crystal sub-elements, voxel-centre sources).  One step = the matrix block of one
z-plane of voxels for all 4096 crystals (37.7 M elements).  Steps alternate between the two
centre planes (15 and 16), the planes the reference arm times in full; with N ranks, rank r
alternates planes 15 + r and 15 + N + r (weak scaling, no data-path collective).  Synthetic,
seeded geometry (the reference ships no parameter files).

Reported: `value` = device-timed elements/s over all ranks (inputs resident in HBM), `e2e`
= the same through the reference-compatible C ABI (PESysMatGen with host buffers: every call
uploads its parameter arrays, since consecutive calls alternate planes, and reads the matrix
back), `roofline` of the PE kernel against measured FP32 / MUFU peaks, `cpu_baseline` = the
FP64 oracle loop (the reference's program restated in C, OpenMP) on a fixed sample, with its
FP32 twin's rate on the same sample beside it, `accuracy` = max / median relative error of
every matrix below against the FP64 oracle on samples, `scatter` = the primary-Compton
rate on a configuration-3 plane (kernel, pair-table preparation, and end to end through
the reference-compatible scatter() with host buffers and bitmap files), `scatter_config2` =
the same on a configuration-2 voxel row, `scatter_grid` = configuration 3 as stated (scatter
points on a 0.25 mm grid inside the crystals and the tungsten, FP64 sums), `batch` = the configuration-4 design sweep in one
batched launch against one launch per task, `sampled` = configuration 2 with the sampling it
states (2x2x2 voxel sub-samples, 2x8x2 crystal sub-elements), in the reference's float
program and (`sampled.local`) in the local-coordinate FP32 form, `fp64` = the FP64 mode (the
element program in double) on the headline plane, `local` = the local-coordinate FP32 mode
(within 1e-5 of FP64) on the same plane.

`--impl reference` times the reference's own CUDA program (its source compiled for sm_100a
by oracle/Makefile into oracle/_ref) through its own host entry points (PESysMatGen,
scatter) on the same elements: strips that together cover planes 15 and 16 exactly once in
the timed steps; the reference has no CPU implementation.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gpu-based-system-matrix-calculation-for-spect-pet_b200")


def _load(name, path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


geometry = _load("sysmat_geometry", os.path.join(PKG, "geometry.py"))
sharding = _load("sysmat_sharding", os.path.join(PKG, "sharding.py"))
roofline_model = _load("sysmat_roofline", os.path.join(PKG, "roofline.py"))

METRIC = "matrix elements/s (PE, scatter)"
UNIT = "elements/s"

# fixed accuracy / CPU-baseline sample of the headline plane: every 16th crystal x the
# voxel row iy = 48 of z-plane 16 (256 x 96 elements)
SAMPLE_DET_STRIDE = 16
SAMPLE_ROW = 48


# ---------------------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sms, maxs, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sms.append(float(p[1]))
                maxs.append(float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxs), "reasons": sorted(reasons),
                "samples": len(sms)}


# ---------------------------------------------------------------------------------------
# distributed plumbing (one process per GPU, NCCL; only timing crosses ranks)

def dist_setup(ngpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != ngpus and world > 1:
        raise SystemExit(f"--gpus {ngpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------------
# workload

def workload(name):
    """(geometry, planes of the image, first headline plane, description)."""
    if name == "config2":
        g = geometry.config2()
        return g, 32, 15, ("config2 PE: 96x96x32 voxels (1 mm), 48x48 hex holes (d 1.5 mm, pitch 2 mm) "
                           "in 20 mm W, 64x64 NaI 1.6x1.6x6 mm; step = one z-plane x 4096 crystals "
                           "(37.7 M elements), z-planes 15 and 16 alternately; 8x16x8 crystal "
                           "sub-elements, voxel-centre sources")
    if name == "config3":
        g = geometry.config3()
        return g, 16, 7, ("config3 PE: 48x48x16 voxels (2 mm), 32x32 holes (d 1 mm) in 10 mm W, "
                          "32x32 NaI 2x2x6 mm; step = one z-plane x 1024 crystals, z-planes 7 and 8 "
                          "alternately")
    if name == "config1":
        g = geometry.config1()
        return g, 1, 0, "config1 PE: 32x32x1 voxels, 7x7 holes, 16x16 NaI"
    raise SystemExit(f"unknown workload {name}")


def step_plane(step, rank, world, n_planes, first):
    """Plane of `rank` at `step`: two planes per rank, taken alternately."""
    if n_planes == 1:
        return 0
    return sharding.plane_for_step(step % 2, rank, world, n_planes, first)


def plane_geometry(g, n_planes, plane):
    return geometry.voxel_slab(g, plane) if n_planes > 1 else g


def rel_err_stats(a, b, scale=None, threshold=1e-5):
    """max / median of |a - b| / max(|b|, tau), tau = 1e-6 * the matrix's largest element
    (`scale`; the sample's own largest when not given), and the count of elements above
    `threshold`."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    m = float(scale) if scale is not None else (np.abs(b).max() if b.size else 0.0)
    tau = 1e-6 * m if m > 0 else 1e-300
    r = np.abs(a - b) / np.maximum(np.abs(b), tau)
    return {"max_rel_err": float(r.max()), "median_rel_err": float(np.median(r)),
            "above_1e-5": int(np.sum(r > threshold)), "elements": int(r.size)}


def scratch_dir(nbytes):
    """A directory with room for `nbytes` of bitmap files (shared memory first), or None."""
    for base in ("/dev/shm", tempfile.gettempdir()):
        try:
            if os.path.isdir(base) and shutil.disk_usage(base).free > nbytes * 1.2 + (1 << 30):
                return tempfile.mkdtemp(prefix="sysmat_bench_", dir=base)
        except OSError:
            continue
    return None


def remove_dir(path):
    if path and os.path.isdir(path):
        for f in os.listdir(path):
            os.remove(os.path.join(path, f))
        os.rmdir(path)


def pinned(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory()
    return t.numpy(), t


def bitmap_bytes(g):
    D = g.n_det
    return 4 * ((D * (D + 1) // 2 * D + 31) // 32 + (g.n_holes_layer0 * D * D + 31) // 32)


# ---------------------------------------------------------------------------------------
# our implementation

def run_sysmat(args, rank, world, local):
    import torch
    sysmat = _load("sysmat_binding", os.path.join(PKG, "sysmat.py"))
    g, n_planes, first, desc = workload(args.workload)
    ctx = sysmat.Context(g, device=local)
    nxy = int(g.image[0]) * int(g.image[1])
    D = ctx.n_det if args.det_count is None else min(args.det_count, ctx.n_det)
    out = torch.empty((D, nxy), dtype=torch.float32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    stream = torch.cuda.current_stream()

    def step(k, events=None):
        plane = step_plane(k, rank, world, n_planes, first)
        flush.fill_(float(k))
        if events:
            events[0].record(stream)
        ctx.pe(out, rotation=0.0, det_count=D, vox_begin=plane * nxy, vox_count=nxy,
               mode=sysmat.MODE_REFERENCE, stream=stream)
        if events:
            events[1].record(stream)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        t0.record(stream)
        for k in range(args.steps):
            step(args.warmup + k, evs[k])
        t1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    region_ms = t0.elapsed_time(t1)
    kernel_ms = [a.elapsed_time(b) for a, b in evs]
    region_ms = max_over_ranks(region_ms, world)
    elements = float(D) * nxy * args.steps * world
    value = elements / (region_ms * 1e-3)

    # roofline: algorithmic work of the timed steps from the kernel's work counters
    fp32_peak, mufu_peak = sysmat.measure_peaks()
    flops = mufu = 0.0
    planes = sorted({step_plane(args.warmup + k, rank, world, n_planes, first) for k in range(args.steps)})
    per_plane = {}
    for p in planes:
        counts = ctx.pe_work(out, det_count=D, vox_begin=p * nxy, vox_count=nxy)
        per_plane[p] = (counts,) + roofline_model.pe_work(counts, n_layers=ctx.n_layers)
    for k in range(args.steps):
        _, f, m = per_plane[step_plane(args.warmup + k, rank, world, n_planes, first)]
        flops += f / args.steps
        mufu += m / args.steps
    k_ms = statistics.mean(kernel_ms)
    ach_f = flops / (k_ms * 1e-3) / 1e12
    ach_m = mufu / (k_ms * 1e-3) / 1e12
    frac_f, frac_m = ach_f / fp32_peak, ach_m / mufu_peak
    traffic = roofline_model.pe_traffic_per_launch(D * nxy)
    if frac_m > frac_f:
        roof = {"bound": "mufu", "achieved": ach_m, "peak": mufu_peak, "unit": "Tops/s", "frac": frac_m}
    else:
        roof = {"bound": "fp32", "achieved": ach_f, "peak": fp32_peak, "unit": "TFLOP/s", "frac": frac_f}
    counts0 = per_plane[planes[0]][0]
    roof.update(traffic=traffic["bytes"] if traffic else None,
                traffic_source=traffic["source"] if traffic else "no DRAM capture summarised",
                algorithmic_bytes=4.0 * D * nxy,
                peak_source="measured on this device by sysmat_measure_peaks (FMA chain, ex2 chain)",
                fp32=dict(achieved=ach_f, peak=fp32_peak, frac=frac_f),
                mufu=dict(achieved=ach_m, peak=mufu_peak, frac=frac_m),
                kernel_ms=k_ms, work_per_launch=dict(flops=flops, mufu_ops=mufu),
                counters=dict(plane=planes[0], **counts0))

    # the accuracy sample's plane, kept for the checker
    acc_plane = first + 1 if n_planes > 1 else 0
    ctx.pe(out, rotation=0.0, det_count=D, vox_begin=acc_plane * nxy, vox_count=nxy, stream=stream)
    torch.cuda.synchronize()
    keep = {"pe": out[:, SAMPLE_ROW * int(g.image[0]):(SAMPLE_ROW + 1) * int(g.image[0])].cpu().numpy()
            if n_planes > 1 else out.cpu().numpy(), "plane": acc_plane, "D": D,
            "pe_max": float(out.max().item())}
    del out, flush
    ctx.close()

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, sysmat, g, rank, world, n_planes, first)

    legs = {}
    if world > 1 and not args.no_scatter:
        legs["scatter_columns"] = run_scatter_columns(args, sysmat, torch, rank, world)
    if world == 1:
        if not args.no_scatter:
            legs["scatter"] = run_scatter(args, sysmat, torch, keep)
        if not args.no_scatter2:
            legs["scatter_config2"] = run_scatter_config2(args, sysmat, torch)
        if not args.no_grid:
            legs["scatter_grid"] = run_scatter_grid(args, sysmat, torch, keep)
        if not args.no_batch:
            legs["batch"] = run_batch(args, sysmat, torch)
            legs["batch_scatter"] = run_batch_scatter(args, sysmat, torch)
        if not args.no_sampled:
            legs["sampled"] = run_sampled(args, sysmat, torch, keep)
        if not args.no_fp64:
            legs["fp64"] = run_fp64(args, sysmat, torch, keep)
        if not args.no_local:
            legs["local"] = run_local(args, sysmat, torch, keep)

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": region_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded geometry)",
        "config": {"workload": desc if D == g.n_det else f"{desc}; first {D} crystals only",
                   "parallelism": f"planes x{world}" if world > 1 else "1 GPU",
                   "planes_timed": planes,
                   "elements_per_step_per_gpu": D * nxy, "summation": "reference order (float chain)",
                   "l2": "flushed between steps (256 MB write)"},
        "clocks": clk.summary(), "gpu_launches": args.steps,
        "roofline": roof, "e2e": e2e,
    }
    result.update(legs)
    return result, keep


def run_e2e(args, sysmat, g, rank, world, n_planes, first):
    """PESysMatGen (the reference-compatible C ABI) with pinned host buffers: parameter
    arrays in, the whole plane's matrix out.  Consecutive calls alternate the two planes, so
    every call uploads its parameter arrays (the library re-uses a device copy only for
    unchanged parameters)."""
    import torch
    steps = min(args.steps, args.e2e_steps)
    geos = [plane_geometry(g, n_planes, step_plane(k, rank, world, n_planes, first)) for k in range(2)]
    nel = geos[0].n_det * geos[0].n_vox
    dst, dst_t = pinned(np.zeros(nel, np.float32))
    pins = [[pinned(a) for a in (gg.collimator, gg.detector, gg.image)] for gg in geos]
    host = [[p[0] for p in pp] for pp in pins]
    dev = torch.cuda.current_device()
    sysmat.PESysMatGen(*host[1], dst, dev)                 # warm-up (the other plane)
    barrier(world)
    t = time.perf_counter()
    for k in range(steps):
        sysmat.PESysMatGen(*host[k % 2], dst, dev)
    dt = time.perf_counter() - t
    barrier(world)
    dt = max_over_ranks(dt, world)
    h2d = 4 * (80000 + 80000 + 100)
    return {"value": nel * steps * world / dt, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": 4 * nel, "steps": steps, "warmup": 1,
            "api": "PESysMatGen (reference-compatible C ABI, pinned host buffers; planes alternate, "
                   "so every call uploads its parameters)"}


def _events(torch, fn, n=1, stream=None):
    stream = stream or torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(n):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / n


def scatter_legacy_e2e(sysmat, g, pe_host, workdir, steps=1):
    """Reference-compatible scatter() (combined program) with host buffers: an untimed call
    computes the relationship bitmaps and writes their files (physics[8] = physics[9] = 1),
    the timed calls read them back (physics[8] = physics[9] = 0), as the rotation loop of
    the reference program does.  Returns seconds per call."""
    import torch
    fc = os.path.join(workdir, "GeometryRelationShip_Crystal2Crystal")
    fh = os.path.join(workdir, "GeometryRelationShip_Collimator2Crystal")
    phys = g.physics.copy()
    phys[8] = phys[9] = 1.0
    pe_p, _t1 = pinned(pe_host.reshape(-1))
    dst, _t2 = pinned(np.zeros(g.n_det * g.n_vox, np.float32))
    dev = torch.cuda.current_device()
    sysmat.scatter(g.collimator, g.detector, g.image, phys, pe_p, fc, fh, dst, dev)
    phys[8] = phys[9] = 0.0
    sysmat.scatter(g.collimator, g.detector, g.image, phys, pe_p, fc, fh, dst, dev)   # warm cache
    t = time.perf_counter()
    for _ in range(steps):
        sysmat.scatter(g.collimator, g.detector, g.image, phys, pe_p, fc, fh, dst, dev)
    return (time.perf_counter() - t) / steps, dst


def run_scatter(args, sysmat, torch, keep):
    """Configuration 3, z-plane 8: 1024 crystals x 2304 voxels, 1024 layer-0 holes."""
    g = geometry.voxel_slab(geometry.config3(), 8)
    ctx = sysmat.Context(g)
    pe = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    ctx.pe(pe)
    bitmaps = {}
    bitmap_ms = _events(torch, lambda: bitmaps.update(c=ctx.bitmap_crystal(), h=ctx.bitmap_collimator()))
    prep_ms = _events(torch, lambda: ctx.scatter_prepare(bitmaps["c"], bitmaps["h"]))
    out = torch.empty_like(pe)
    ctx.scatter(out, pe)
    ms = _events(torch, lambda: ctx.scatter(out, pe), n=3)
    nel = ctx.n_det * ctx.n_vox
    res = {"value": nel / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
           "prepare_ms": prep_ms, "bitmaps_ms": bitmap_ms,
           "value_with_prepare": nel / ((ms + prep_ms) * 1e-3),
           "workload": "config3 primary Compton (crystal + collimator) on z-plane 8: 1024 crystals x "
                       "2304 voxels, 1024 layer-0 holes; value = scatter kernel on resident buffers, "
                       "value_with_prepare adds the pair-table preparation"}
    keep["scatter"] = {"geo": g, "pe": pe.cpu().numpy(), "out": out.cpu().numpy(), "max": float(out.max().item()),
                       "bc": bitmaps["c"].cpu().numpy().view(np.uint32),
                       "bh": bitmaps["h"].cpu().numpy().view(np.uint32)}
    del bitmaps
    ctx.close()
    if not args.no_e2e:
        work = scratch_dir(bitmap_bytes(g))
        try:
            if work is None:
                res["e2e"] = {"unavailable": "no scratch space for the bitmap files"}
            else:
                s, _ = scatter_legacy_e2e(sysmat, g, keep["scatter"]["pe"], work)
                res["e2e"] = {"value": nel / s, "unit": UNIT, "ms_per_step": s * 1e3,
                              "h2d_bytes_per_step": 4 * nel + bitmap_bytes(g) + 4 * 160200,
                              "d2h_bytes_per_step": 4 * nel,
                              "api": "scatter() (reference-compatible C ABI, combined program): "
                                     "bitmap files read, PE uploaded, pair tables built, scatter "
                                     "matrix read back, all inside the timed call"}
        finally:
            remove_dir(work)
    return res


def run_scatter_grid(args, sysmat, torch, keep):
    """Configuration 3 as stated: primary Compton scatter with scatter points on a 0.25 mm grid
    inside the crystals (1024 x 8 x 24 x 8 cells) and the tungsten (256 x 40 x 256 cells of the
    plate, minus the holes), FP64 sums per element (sysmat_scatter_grid).  Voxel row 24 of
    z-plane 8 (48 voxels) x 1024 crystals per step; one untimed step, one timed."""
    g = geometry.voxel_slab(geometry.config3(), 8, 24, 1)
    ctx = sysmat.Context(g)
    out = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    ctx.scatter_grid(out, cell=0.25)
    ms = _events(torch, lambda: ctx.scatter_grid(out, cell=0.25))
    keep["scatter_grid"] = {"geo": g, "out": out.cpu().numpy(), "max": float(out.max().item())}
    nel = ctx.n_det * ctx.n_vox
    ctx.close()
    return {"value": nel / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "summation": "FP64 per element",
            "workload": "config3 grid scatter: scatter points on a 0.25 mm grid inside the crystals and the "
                        f"collimator's tungsten; voxel row 24 of z-plane 8 x 1024 crystals ({nel} elements)"}


def run_scatter_columns(args, sysmat, torch, rank, world):
    """Configuration 3, z-plane 8 (1024 crystals x 2304 voxels, crystal + collimator parts),
    split across ranks by voxel columns (sharding.voxel_block): each rank computes the PE
    columns its scatter columns read, so the ranks exchange nothing (strong scaling of one
    plane; device time, max over ranks)."""
    g = geometry.voxel_slab(geometry.config3(), 8)
    ctx = sysmat.Context(g)
    ctx.scatter_prepare(ctx.bitmap_crystal(), ctx.bitmap_collimator())
    v0, nv = sharding.voxel_block(ctx.n_vox, rank, world)
    pe = torch.zeros((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    out = torch.empty((ctx.n_det, nv), dtype=torch.float32, device="cuda")

    def step():
        ctx.scatter_columns(out, v0, nv, pe=pe)

    step()
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(_events(torch, step, n=2), world)
    ctx.close()
    nel = ctx.n_det * ctx.n_vox
    return {"value": nel / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "scaling": "strong",
            "workload": f"config3 z-plane 8 ({nel} elements) PE columns + crystal and collimator scatter, voxel "
                        f"columns split over {world} ranks, no exchange"}


def config2_scatter_slab():
    """Configuration 2 scatter sample: voxel row iy = 48 of z-plane 16 (96 voxels) x 4096
    crystals, 2304 layer-0 holes."""
    return geometry.voxel_slab(geometry.config2(), 16, SAMPLE_ROW, 1)


def run_scatter_config2(args, sysmat, torch):
    g = config2_scatter_slab()
    ctx = sysmat.Context(g)
    pe = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    ctx.pe(pe)
    bitmaps = {}
    bitmap_ms = _events(torch, lambda: bitmaps.update(c=ctx.bitmap_crystal(), h=ctx.bitmap_collimator()))
    prep_ms = _events(torch, lambda: ctx.scatter_prepare(bitmaps["c"], bitmaps["h"]))
    del bitmaps
    out = torch.empty_like(pe)
    ctx.scatter(out, pe)
    ms = _events(torch, lambda: ctx.scatter(out, pe), n=2)
    nel = ctx.n_det * ctx.n_vox
    pe_h = pe.cpu().numpy()
    ctx.close()
    del pe, out
    torch.cuda.empty_cache()
    res = {"value": nel / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "prepare_ms": prep_ms,
           "bitmaps_ms": bitmap_ms, "value_with_prepare": nel / ((ms + prep_ms) * 1e-3),
           "workload": "config2 primary Compton (crystal + collimator): voxel row 48 of z-plane 16 "
                       "(96 voxels) x 4096 crystals, 2304 layer-0 holes"}
    if not args.no_e2e:
        work = scratch_dir(bitmap_bytes(g))
        try:
            if work is None:
                res["e2e"] = {"unavailable": "no scratch space for the bitmap files"}
            else:
                s, _ = scatter_legacy_e2e(sysmat, g, pe_h, work)
                res["e2e"] = {"value": nel / s, "unit": UNIT, "ms_per_step": s * 1e3,
                              "h2d_bytes_per_step": 4 * nel + bitmap_bytes(g) + 4 * 160200,
                              "d2h_bytes_per_step": 4 * nel,
                              "api": "scatter() with host buffers, bitmap files read inside the call"}
        finally:
            remove_dir(work)
    return res


def run_sampled(args, sysmat, torch, keep, rows=512):
    """Configuration 2 with the sampling it states (no reference counterpart): each voxel
    sampled at 2x2x2 source points, each crystal divided 2x8x2 (x, depth, z), every
    contribution summed in FP64 (sysmat_pe_sampled).  `rows` crystals of the array's centre x
    z-plane 16 (9216 voxels) per step."""
    g = geometry.config2()
    ctx = sysmat.Context(g)
    nxy = int(g.image[0]) * int(g.image[1])
    d0 = ctx.n_det // 2 - rows // 2
    out = torch.empty((rows, nxy), dtype=torch.float32, device="cuda")

    def step(mode):
        ctx.pe_sampled(out, (2, 8, 2), (2, 2, 2), det_begin=d0, det_count=rows, vox_begin=16 * nxy, vox_count=nxy,
                       mode=mode)

    nx = int(g.image[0])
    res = {}
    for key, mode in (("sampled", sysmat.MODE_PRECISE), ("sampled_local", sysmat.MODE_LOCAL)):
        step(mode)
        ms = _events(torch, lambda: step(mode), n=2)
        keep[key] = {"d0": d0, "out": out[:, SAMPLE_ROW * nx:(SAMPLE_ROW + 1) * nx].cpu().numpy(),
                     "max": float(out.max().item())}
        res[key] = {"value": rows * nxy / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "rays_per_element": 8 * 32,
                    "arithmetic": "f32, FP64 sums" if key == "sampled" else "f32 (local), compensated sums",
                    "workload": f"config2 as stated: 2x2x2 voxel sub-samples, 2x8x2 crystal sub-elements; crystals "
                                f"{d0}..{d0 + rows - 1} x z-plane 16 ({rows * nxy} elements)"}
    ctx.close()
    res["sampled"]["local"] = res.pop("sampled_local")
    return res["sampled"]


def run_fp64(args, sysmat, torch, keep):
    """FP64 mode (the reference's element program in double: within the float output's
    rounding of the FP64 restatement) on z-plane 16 of configuration 2 for all 4096
    crystals, reference sampling (8x16x8, voxel centres); one untimed step, one timed."""
    g = geometry.config2()
    ctx = sysmat.Context(g)
    nxy = int(g.image[0]) * int(g.image[1])
    D = ctx.n_det if args.fp64_crystals is None else min(args.fp64_crystals, ctx.n_det)
    d0 = (ctx.n_det - D) // 2
    out = torch.empty((D, nxy), dtype=torch.float32, device="cuda")

    def step():
        ctx.pe(out, det_begin=d0, det_count=D, vox_begin=16 * nxy, vox_count=nxy, mode=sysmat.MODE_FP64)

    step()
    ms = _events(torch, step)
    nx = int(g.image[0])
    keep["fp64"] = {"d0": d0, "out": out[:, SAMPLE_ROW * nx:(SAMPLE_ROW + 1) * nx].cpu().numpy()}
    ctx.close()
    return {"value": D * nxy / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "arithmetic": "f64",
            "workload": f"config2 PE in FP64: crystals {d0}..{d0 + D - 1} x z-plane 16 ({D * nxy} elements)"}


def run_local(args, sysmat, torch, keep):
    """Local-coordinate FP32 mode (the reference's element program in float arithmetic that
    stays within 1e-5 of its FP64 evaluation) on z-plane 16 of configuration 2, all 4096
    crystals, reference sampling; one untimed step, two timed."""
    g = geometry.config2()
    ctx = sysmat.Context(g)
    nxy = int(g.image[0]) * int(g.image[1])
    D = ctx.n_det if args.det_count is None else min(args.det_count, ctx.n_det)
    out = torch.empty((D, nxy), dtype=torch.float32, device="cuda")

    def step():
        ctx.pe(out, det_count=D, vox_begin=16 * nxy, vox_count=nxy, mode=sysmat.MODE_LOCAL)

    step()
    ms = _events(torch, step, n=2)
    nx = int(g.image[0])
    if D == ctx.n_det:
        keep["local"] = {"d0": 0, "out": out[:, SAMPLE_ROW * nx:(SAMPLE_ROW + 1) * nx].cpu().numpy()}
    ctx.close()
    what = "all crystals" if D == ctx.n_det else f"crystals 0..{D - 1}"
    return {"value": D * nxy / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "arithmetic": "f32 (local)",
            "workload": f"config2 PE, local-coordinate FP32 mode: {what} x z-plane 16 ({D * nxy} elements)"}


def run_batch(args, sysmat, torch, n_instances=64, rows=8, sweep=True):
    """Design sweep of configuration 4: every instance x every one of its rotations, each task
    a block of `rows` crystals (centre of the 32x32 array) x one z-plane (1024 voxels).  The
    batched form (one autotuned persistent launch, replayed as a CUDA graph) against the plain
    form (one sysmat_pe call per instance and rotation), same outputs."""
    geos = geometry.config4(n_instances=n_instances)
    ctxs = [sysmat.Context(gg) for gg in geos]
    d0, v0, nv = 16 * 32 + 16 - rows // 2, 1024 * 8, 1024
    tasks = [(k, float(r), d0, rows, v0, nv) for k, gg in enumerate(geos) for r in range(gg.n_rot)]
    out = torch.empty((len(tasks), rows, nv), dtype=torch.float32, device="cuda")
    plan = sysmat.BatchPlan(ctxs, [t + (out[i],) for i, t in enumerate(tasks)])
    stream = torch.cuda.current_stream()
    tiles = plan.tune(stream=stream)
    plan.run(stream=stream)                                   # capture + warm-up
    batch_ms = _events(torch, lambda: plan.run(stream=stream), n=2, stream=stream)
    ref = out.clone()

    def plain():
        for i, (k, r, dd, nd, vv, nn) in enumerate(tasks):
            ctxs[k].pe(out[i], rotation=r, det_begin=dd, det_count=nd, vox_begin=vv, vox_count=nn,
                       stream=stream)

    plain()                                                   # warm-up
    plain_ms = _events(torch, plain, stream=stream)
    same = bool(torch.equal(out, ref))
    plan.close()
    nel = len(tasks) * rows * nv
    by_rows = None
    if sweep:
        # the batched form's gain against per-task calls as the tasks grow (16 designs)
        by_rows = {}
        for r in (2, 32):
            sub = run_batch(args, sysmat, torch, n_instances=16, rows=r, sweep=False)
            by_rows[str(r)] = {"speedup_vs_plain": sub["speedup_vs_plain"], "tasks": sub["tasks"],
                               "elements_per_step": sub["elements_per_step"]}
    return {"value": nel / (batch_ms * 1e-3), "unit": UNIT, "ms_per_step": batch_ms,
            "plain_value": nel / (plain_ms * 1e-3), "plain_ms_per_step": plain_ms,
            "speedup_vs_plain": plain_ms / batch_ms, "outputs_identical": same,
            "tiles": list(tiles), "tasks": len(tasks), "elements_per_step": nel,
            "gpu_launches_per_step": {"batched": 1, "plain": len(tasks)},
            "speedup_by_rows_per_task": by_rows,
            "workload": f"config4 design sweep: {n_instances} seeded collimators x their 12-60 rotations "
                        f"({len(tasks)} tasks), each crystals {d0}..{d0 + rows - 1} x z-plane 8 "
                        f"(1024 voxels)"}


def run_batch_scatter(args, sysmat, torch, n_instances=16, n_rot=4, rows=8):
    """Batched scatter on a configuration-4 design sweep: n_instances seeded collimators x their
    first n_rot rotations, each task the crystal + collimator scatter of `rows` crystals (centre
    of the 32x32 array) x z-plane 8 (1024 voxels), reading that rotation's PE columns.  One
    persistent launch (replayed as a CUDA graph) against one sysmat_scatter launch per task,
    same outputs.  Pair tables and PE matrices are built outside the timed region."""
    geos = geometry.config4(n_instances=n_instances)
    ctxs = [sysmat.Context(gg) for gg in geos]
    d0, v0, nv = 16 * 32 + 16 - rows // 2, 1024 * 8, 1024
    items, pes = [], []
    for k, ctx in enumerate(ctxs):
        bc, bh = ctx.bitmap_crystal(), ctx.bitmap_collimator()
        ctx.scatter_prepare(bc, bh)
        del bc, bh
        for r in range(min(n_rot, geos[k].n_rot)):
            pe = torch.zeros((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
            ctx.pe(pe[:, v0:v0 + nv], rotation=float(r), vox_begin=v0, vox_count=nv)
            pes.append(pe)
            out = torch.empty((rows, nv), dtype=torch.float32, device="cuda")
            items.append((k, 3, sysmat.HOLE_MODEL_COMBINED, float(r), pe, d0, rows, v0, nv, out))
    stream = torch.cuda.current_stream()
    plan = sysmat.ScatterBatchPlan(ctxs, items, stream=stream)
    plan.run(stream=stream)                                   # capture + warm-up
    batch_ms = _events(torch, lambda: plan.run(stream=stream), n=3, stream=stream)
    ref = [it[-1].clone() for it in items]

    def plain():
        for (k, parts, model, rot, pe, dd, nd, vv, nn, out) in items:
            ctxs[k].scatter(out, pe, parts=parts, hole_model=model, rotation=rot, det_begin=dd, det_count=nd,
                            vox_begin=vv, vox_count=nn, stream=stream)

    plain()
    plain_ms = _events(torch, plain, n=3, stream=stream)
    same = all(bool(torch.equal(it[-1], r)) for it, r in zip(items, ref))
    plan.close()
    nel = len(items) * rows * nv
    for c in ctxs:
        c.close()
    return {"value": nel / (batch_ms * 1e-3), "unit": UNIT, "ms_per_step": batch_ms,
            "plain_value": nel / (plain_ms * 1e-3), "plain_ms_per_step": plain_ms,
            "speedup_vs_plain": plain_ms / batch_ms, "outputs_identical": same, "tasks": len(items),
            "gpu_launches_per_step": {"batched": 1, "plain": len(items)},
            "workload": f"config4 design sweep, scatter: {n_instances} seeded collimators x {n_rot} rotations, each "
                        f"task crystals {d0}..{d0 + rows - 1} x z-plane 8 (1024 voxels), crystal + collimator parts"}


# ---------------------------------------------------------------------------------------
# CPU baseline and accuracy: the oracle (reference arithmetic in C, FP32 and FP64) on the
# host cores, as the checker of the matrices the GPU legs produced

def sample_rows(g):
    return np.arange(SAMPLE_DET_STRIDE // 2, g.n_det, SAMPLE_DET_STRIDE)


def cpu_baseline(args, g, n_planes, keep):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    plane = keep["plane"]
    gp = plane_geometry(g, n_planes, plane)
    nx = int(g.image[0])
    v0, nv = (nx * SAMPLE_ROW, nx) if n_planes > 1 else (0, g.n_vox)
    rows = sample_rows(g)
    rows = rows[rows < keep["D"]]
    t = time.perf_counter()
    o64 = oracle.pe(gp, prec=64, dets=rows, v0=v0, nv=nv, threads=threads)
    dt = time.perf_counter() - t
    t = time.perf_counter()
    o32 = oracle.pe(gp, prec=32, dets=rows, v0=v0, nv=nv, threads=threads)
    dt32 = time.perf_counter() - t
    el = rows.size * nv
    base = {"value": el / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "fp32_twin_value": el / dt32,
            "sample": f"{rows.size} crystals (every {SAMPLE_DET_STRIDE}th) x {nv} voxels (voxel row "
                      f"{SAMPLE_ROW} of z-plane {plane}); FP64 oracle, OpenMP, {dt:.1f} s (FP32 twin on the "
                      f"same elements: {dt32:.1f} s)"}
    pe_gpu = keep["pe"][rows]
    scale = keep["pe_max"]                      # the plane's largest element: tau = 1e-6 of it
    acc = {"pe": dict(rel_err_stats(pe_gpu, o64, scale), vs="FP64 oracle",
                      mode="reference (the reference's float program)",
                      bit_identical_to_fp32_twin=float(np.mean(pe_gpu == o32.astype(np.float32))),
                      sample=base["sample"])}
    if "fp64" in keep:
        f = keep["fp64"]
        sel = rows[(rows >= f["d0"]) & (rows < f["d0"] + f["out"].shape[0])]
        idx = np.searchsorted(rows, sel)
        acc["fp64"] = dict(rel_err_stats(f["out"][sel - f["d0"]], o64[idx], scale), vs="FP64 oracle",
                           sample=f"{sel.size} of the crystals above x the same voxel row")
    if "local" in keep:
        f = keep["local"]
        acc["local"] = dict(rel_err_stats(f["out"][rows], o64, scale), vs="FP64 oracle", sample=base["sample"])
    if "sampled" in keep:
        s = keep["sampled"]
        sel = np.arange(s["d0"] + 8, s["d0"] + s["out"].shape[0], 128)
        gs = geometry.voxel_slab(g, 16)
        os64 = oracle.pe_sampled(gs, (2, 8, 2), (2, 2, 2), prec=64, dets=sel, v0=nx * SAMPLE_ROW, nv=nx,
                                 threads=threads)
        acc["sampled"] = dict(rel_err_stats(s["out"][sel - s["d0"]], os64, s["max"]), vs="FP64 oracle (sampled form)",
                              sample=f"crystals {sel.tolist()} x voxel row {SAMPLE_ROW} of z-plane 16")
        if "sampled_local" in keep:
            s = keep["sampled_local"]
            acc["sampled_local"] = dict(rel_err_stats(s["out"][sel - s["d0"]], os64, s["max"]),
                                        vs="FP64 oracle (sampled form)",
                                        sample=f"crystals {sel.tolist()} x voxel row {SAMPLE_ROW} of z-plane 16")
    if "scatter" in keep:
        s = keep["scatter"]
        gs = s["geo"]
        nx3 = int(gs.image[0])
        sel = np.arange(64, gs.n_det, 128)
        v3 = nx3 * 24
        o = oracle.scatter(gs, s["pe"], "crystal", s["bc"], prec=64, dets=sel, v0=v3, nv=nx3, threads=threads)
        o += oracle.scatter(gs, s["pe"], "collimator", s["bh"], prec=64, dets=sel, v0=v3, nv=nx3,
                            threads=threads)
        acc["scatter"] = dict(rel_err_stats(s["out"][sel][:, v3:v3 + nx3], o, s["max"]), vs="FP64 oracle",
                              sample=f"crystals {sel.tolist()} x voxel row 24 of config3 z-plane 8 "
                                     "(the GPU's PE matrix and bitmaps as input)")
    if "scatter_grid" in keep:
        s = keep["scatter_grid"]
        d, v = 528, 22
        o = oracle.scatter_grid(s["geo"], parts=3, cell=0.25, dets=[d], v0=v, nv=1, threads=threads)
        acc["scatter_grid"] = dict(rel_err_stats(s["out"][d:d + 1, v:v + 1], o, s["max"]),
                                   vs="FP64 definition of the grid model",
                                   sample=f"crystal {d} x voxel {v} of the grid leg's voxel row")
    return base, acc


# ---------------------------------------------------------------------------------------
# reference arm: the reference's own CUDA program through its own host entry points

def reference_strips(n_rows, planes, steps):
    """Strips (plane, iy0, ny) of each timed step: together they cover every voxel row of
    `planes` exactly once."""
    total = n_rows * len(planes)
    out = []
    for k in range(steps):
        a, b = (k * total) // steps, ((k + 1) * total) // steps
        parts = []
        while a < b:
            p, iy = divmod(a, n_rows)
            n = min(b - a, n_rows - iy)
            parts.append((planes[p], iy, n))
            a += n
        out.append(parts)
    return out


def run_reference(args, rank, world, local):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_lib
    g, n_planes, first, desc = workload(args.workload)
    if rank != 0:
        return None
    if not ref_lib.available():
        return {"impl": "reference", "unavailable": "oracle/_ref not built (make -C oracle ref)"}
    ny = int(g.image[1])
    nx = int(g.image[0])
    planes = [first, first + 1] if n_planes > 1 else [0]
    strips = reference_strips(ny, planes, args.steps) if n_planes > 1 else [[(0, 0, ny)]] * args.steps
    warm = [[(planes[-1], k % ny, 1)] for k in range(args.warmup)] if n_planes > 1 else strips[:args.warmup]

    def slab(p, iy0, n):
        return geometry.voxel_slab(g, p, iy0, n) if n_planes > 1 else g

    for parts in warm:
        for p in parts:
            ref_lib.pe(slab(*p), cuda_id=local)
    outs = {}
    nel = 0
    t = time.perf_counter()
    for parts in strips:
        for p in parts:
            gs = slab(*p)
            outs[p] = ref_lib.pe(gs, cuda_id=local)
            nel += gs.n_det * gs.n_vox
    dt = time.perf_counter() - t
    value = nel / dt
    sample = (f"z-planes {planes} x {g.n_det} crystals in {args.steps} strips of voxel rows, each "
              f"row once ({nel} elements), one PESysMatGen call per strip and plane")
    res = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded geometry)",
           "config": {"workload": desc, "sample": sample, "planes_timed": planes,
                      "build": "reference sources compiled for sm_100a (nvcc -O3, oracle/Makefile)"},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                            "sample": sample,
                            "runs_on": "B200: the reference is a CUDA program (it has no CPU "
                                       "implementation of the path); one host thread drives it "
                                       "through its own host entry point"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "gpu_launches": sum(len(p) for p in strips)}
    # the reference's own error against the FP64 oracle on the bench's accuracy sample
    if n_planes > 1 and not args.no_cpu_baseline:
        import oracle
        rows = sample_rows(g)
        acc_plane = first + 1
        got = None
        for (p, iy0, n), o in outs.items():
            if p == acc_plane and iy0 <= SAMPLE_ROW < iy0 + n:
                r = SAMPLE_ROW - iy0
                got = o[rows][:, r * nx:(r + 1) * nx]
        if got is not None:
            gp = geometry.voxel_slab(g, acc_plane)
            o64 = oracle.pe(gp, prec=64, dets=rows, v0=nx * SAMPLE_ROW, nv=nx, threads=os.cpu_count() or 1)
            scale = max(float(o.max()) for (p, _, _), o in outs.items() if p == acc_plane)
            res["accuracy"] = {"pe": dict(rel_err_stats(got, o64, scale), vs="FP64 oracle",
                                          sample=f"{rows.size} crystals (every {SAMPLE_DET_STRIDE}th) x "
                                                 f"voxel row {SAMPLE_ROW} of z-plane {acc_plane}")}
    del outs
    if not args.no_scatter:
        res["scatter"] = run_reference_scatter(ref_lib, local, geometry.voxel_slab(geometry.config3(), 8),
                                               "config3 primary Compton (crystal + collimator), reference "
                                               "combined program, z-plane 8")
    if not args.no_scatter2:
        res["scatter_config2"] = run_reference_scatter(ref_lib, local, config2_scatter_slab(),
                                                       "config2 primary Compton, reference combined program, "
                                                       "voxel row 48 of z-plane 16")
    return res


def run_reference_scatter(ref_lib, local, g, what):
    """The reference's combined scatter program on `g`: a warm-up call computes and writes the
    relationship bitmaps, the timed call reads them back, as a rotation loop of the reference
    program would."""
    work = scratch_dir(bitmap_bytes(g))
    if work is None:
        return {"unavailable": "no scratch space for the bitmap files"}
    try:
        pe = ref_lib.pe(g, cuda_id=local)
        ref_lib.scatter(g, pe, "combined", cuda_id=local, workdir=work)
        t = time.perf_counter()
        ref_lib.scatter(g, pe, "combined", cuda_id=local, workdir=work, load_bitmaps=True)
        dt = time.perf_counter() - t
    finally:
        remove_dir(work)
    nel = g.n_det * g.n_vox
    return {"value": nel / dt, "unit": UNIT, "ms_per_step": dt * 1e3,
            "workload": f"{what}: {g.n_det} crystals x {g.n_vox} voxels, bitmaps read from the files of "
                        "a warm-up call"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sysmat", choices=("sysmat", "reference"))
    ap.add_argument("--workload", default="config2", choices=("config1", "config2", "config3"))
    ap.add_argument("--det-count", type=int, default=None,
                    help="first N crystals only (small cases for profiling)")
    ap.add_argument("--e2e-steps", type=int, default=6, help="timed PESysMatGen calls of the e2e leg (at most --steps)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-scatter", action="store_true")
    ap.add_argument("--no-scatter2", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-sampled", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-local", action="store_true")
    ap.add_argument("--no-grid", action="store_true")
    ap.add_argument("--fp64-crystals", type=int, default=None,
                    help="crystals (centred) of the FP64 leg; default all (profiling uses a small case)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "sysmat":
        args.warmup = 3
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            res = run_reference(args, rank, world, local)
        else:
            res, keep = run_sysmat(args, rank, world, local)
            if rank == 0 and not args.no_cpu_baseline:
                g, n_planes, _, _ = workload(args.workload)
                res["cpu_baseline"], res["accuracy"] = cpu_baseline(args, g, n_planes, keep)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
