#!/usr/bin/env python
"""Benchmark: SPECT system-matrix throughput (matrix elements/s) on B200.

Workload (default): the production photoelectric system of configuration 2 — 96x96x32
voxels of 1 mm, a 20 mm tungsten plate with 48x48 hexagonal holes (1.5 mm, pitch 2 mm),
64x64 NaI crystals of 1.6x1.6x6 mm — with the reference's own integration constants
(8x16x8 crystal sub-elements, voxel-centre sources).  One step = the matrix block of one
z-plane of voxels for all 4096 crystals (37.7 M elements); ranks take interleaved planes
(weak scaling, no data-path collective).  Synthetic, seeded geometry (the reference ships
no parameter files).

Reported: `value` = device-timed elements/s over all ranks (inputs resident in HBM), `e2e`
= the same through the reference-compatible C ABI (PESysMatGen with host buffers, host to
device parameter copy and device to host matrix copy inside the timed region), `roofline`
of the PE kernel against measured FP32 / MUFU peaks, `cpu_baseline` = the FP64 oracle loop
(the reference's program restated in C, OpenMP) on a bounded sample, with its FP32 twin's
rate on the same sample beside it, and `scatter` =
the primary-Compton rate on a configuration-3 plane, `batch` = the configuration-4 design
sweep in one batched launch against one launch per task, `sampled` = configuration 2 with
the sampling it states (2x2x2 voxel sub-samples, 2x8x2 crystal sub-elements), `fp64` = the
FP64 mode (the element program in double) on the headline plane.

`--impl reference` times the reference's own CUDA program (its source compiled for sm_100a
by oracle/Makefile into oracle/_ref) through its own host entry point PESysMatGen on a
bounded sample of the same workload; the reference has no CPU implementation.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
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


def sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------------------
# workload

def workload(name):
    if name == "config2":
        g = geometry.config2()
        return g, 32, ("config2 PE: 96x96x32 voxels (1 mm), 48x48 hex holes (d 1.5 mm, pitch 2 mm) "
                       "in 20 mm W, 64x64 NaI 1.6x1.6x6 mm; step = one z-plane x 4096 crystals "
                       "(37.7 M elements); 8x16x8 crystal sub-elements, voxel-centre sources")
    if name == "config3":
        g = geometry.config3()
        return g, 16, ("config3 PE: 48x48x16 voxels (2 mm), 32x32 holes (d 1 mm) in 10 mm W, "
                       "32x32 NaI 2x2x6 mm; step = one z-plane x 1024 crystals")
    if name == "config1":
        g = geometry.config1()
        return g, 1, "config1 PE: 32x32x1 voxels, 7x7 holes, 16x16 NaI"
    raise SystemExit(f"unknown workload {name}")


def plane_geometry(g, plane):
    return geometry.voxel_slab(g, plane)


# ---------------------------------------------------------------------------------------
# our implementation

def run_sysmat(args, rank, world, local):
    import torch
    sysmat = _load("sysmat_binding", os.path.join(PKG, "sysmat.py"))
    g, n_planes, desc = workload(args.workload)
    first = n_planes // 2 if n_planes > 1 else 0
    ctx = sysmat.Context(g, device=local)
    nxy = int(g.image[0]) * int(g.image[1])
    D = ctx.n_det if args.det_count is None else min(args.det_count, ctx.n_det)
    out = torch.empty((D, nxy), dtype=torch.float32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    stream = torch.cuda.current_stream()

    def step(k, events=None):
        plane = sharding.plane_for_step(k, rank, world, n_planes, first) if n_planes > 1 else 0
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
    kernel_ms = []
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

    # roofline: algorithmic work of one step (plane) from the kernel's work counters
    work_plane = sharding.plane_for_step(args.warmup, rank, world, n_planes, first) if n_planes > 1 else 0
    counts = ctx.pe_work(out, det_count=D, vox_begin=work_plane * nxy, vox_count=nxy)
    fp32_peak, mufu_peak = sysmat.measure_peaks()
    flops, mufu = roofline_model.pe_work(counts, n_layers=ctx.n_layers)
    k_ms = statistics.mean(kernel_ms)
    ach_f = flops / (k_ms * 1e-3) / 1e12
    ach_m = mufu / (k_ms * 1e-3) / 1e12
    frac_f, frac_m = ach_f / fp32_peak, ach_m / mufu_peak
    traffic = roofline_model.measured_traffic("pe_kernel", args.workload)
    if frac_m > frac_f:
        roof = {"bound": "mufu", "achieved": ach_m, "peak": mufu_peak, "unit": "Tops/s", "frac": frac_m}
    else:
        roof = {"bound": "fp32", "achieved": ach_f, "peak": fp32_peak, "unit": "TFLOP/s", "frac": frac_f}
    roof.update(traffic=traffic, peak_source="measured on this device by sysmat_measure_peaks",
                fp32=dict(achieved=ach_f, peak=fp32_peak, frac=frac_f),
                mufu=dict(achieved=ach_m, peak=mufu_peak, frac=frac_m),
                kernel_ms=k_ms, work=dict(flops=flops, mufu_ops=mufu, **counts))

    # end to end through the reference-compatible C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, sysmat, g, rank, world, n_planes, first)

    scatter = None
    if not args.no_scatter and world == 1:
        scatter = run_scatter(args, sysmat, torch)

    batch = None
    if not args.no_batch and world == 1:
        batch = run_batch(args, sysmat, torch)

    sampled = None
    if not args.no_sampled and world == 1:
        sampled = run_sampled(args, sysmat, torch)

    fp64 = None
    if not args.no_fp64 and world == 1:
        fp64 = run_fp64(args, sysmat, torch)

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": region_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded geometry)",
        "config": {"workload": desc if D == g.n_det else f"{desc}; first {D} crystals only",
                   "parallelism": f"planes x{world}" if world > 1 else "1 GPU",
                   "elements_per_step_per_gpu": D * nxy, "summation": "reference order (float chain)",
                   "l2": "flushed between steps (256 MB write)"},
        "clocks": clk.summary(), "gpu_launches": args.steps,
        "roofline": roof, "e2e": e2e, "scatter": scatter, "batch": batch, "sampled": sampled, "fp64": fp64,
    }
    return result


def run_e2e(args, sysmat, g, rank, world, n_planes, first):
    import torch
    geos = []
    for k in range(args.warmup + args.steps):
        plane = sharding.plane_for_step(k, rank, world, n_planes, first) if n_planes > 1 else 0
        geos.append(plane_geometry(g, plane) if n_planes > 1 else g)
    nel = geos[0].n_det * geos[0].n_vox
    dst = torch.empty(nel, dtype=torch.float32).pin_memory().numpy()
    pins = []
    for gg in geos:
        arrs = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory().numpy()
                for a in (gg.collimator, gg.detector, gg.image)]
        pins.append(arrs)
    for k in range(args.warmup):
        sysmat.PESysMatGen(*pins[k], dst, torch.cuda.current_device())
    barrier(world)
    t = time.perf_counter()
    for k in range(args.warmup, args.warmup + args.steps):
        sysmat.PESysMatGen(*pins[k], dst, torch.cuda.current_device())
    dt = time.perf_counter() - t
    barrier(world)
    dt = max_over_ranks(dt, world)
    h2d = 4 * (80000 + 80000 + 100)
    return {"value": nel * args.steps * world / dt, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": 4 * nel, "api": "PESysMatGen (reference-compatible C ABI, host buffers)"}


def run_scatter(args, sysmat, torch):
    g = geometry.voxel_slab(geometry.config3(), 8)
    ctx = sysmat.Context(g)
    pe = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    ctx.pe(pe)
    ctx.scatter_prepare(ctx.bitmap_crystal(), ctx.bitmap_collimator())
    out = torch.empty_like(pe)
    ctx.scatter(out, pe)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = 2
    a.record()
    for _ in range(n):
        ctx.scatter(out, pe)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / n
    return {"value": ctx.n_det * ctx.n_vox / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "workload": "config3 primary Compton (crystal + collimator) on z-plane 8: 1024 crystals x "
                        "2304 voxels, 1024 layer-0 holes"}


def run_sampled(args, sysmat, torch, rows=512):
    """Configuration 2 with the sampling it states (no reference counterpart): each voxel
    sampled at 2x2x2 source points, each crystal divided 2x8x2 (x, depth, z), every
    contribution summed in FP64 (sysmat_pe_sampled).  `rows` crystals of the array's centre x
    z-plane 16 (9216 voxels) per step."""
    g = geometry.config2()
    ctx = sysmat.Context(g)
    nxy = int(g.image[0]) * int(g.image[1])
    d0 = ctx.n_det // 2 - rows // 2
    out = torch.empty((rows, nxy), dtype=torch.float32, device="cuda")

    def step():
        ctx.pe_sampled(out, (2, 8, 2), (2, 2, 2), det_begin=d0, det_count=rows, vox_begin=16 * nxy, vox_count=nxy)

    step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = 2
    a.record()
    for _ in range(n):
        step()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / n
    return {"value": rows * nxy / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "rays_per_element": 8 * 32,
            "summation": "FP64",
            "workload": f"config2 as stated: 2x2x2 voxel sub-samples, 2x8x2 crystal sub-elements; crystals "
                        f"{d0}..{d0 + rows - 1} x z-plane 16 ({rows * nxy} elements)"}


def run_fp64(args, sysmat, torch):
    """FP64 mode (the reference's element program in double: within the float output's
    rounding of the FP64 restatement) on the headline step: z-plane 16 of configuration 2 for
    all 4096 crystals, reference sampling (8x16x8, voxel centres); one untimed step, one timed."""
    g = geometry.config2()
    ctx = sysmat.Context(g)
    nxy = int(g.image[0]) * int(g.image[1])
    D = ctx.n_det if args.fp64_crystals is None else min(args.fp64_crystals, ctx.n_det)
    d0 = (ctx.n_det - D) // 2
    out = torch.empty((D, nxy), dtype=torch.float32, device="cuda")

    def step():
        ctx.pe(out, det_begin=d0, det_count=D, vox_begin=16 * nxy, vox_count=nxy, mode=sysmat.MODE_FP64)

    step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    step()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    return {"value": D * nxy / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "arithmetic": "f64",
            "workload": f"config2 PE in FP64: crystals {d0}..{d0 + D - 1} x z-plane 16 ({D * nxy} elements)"}


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
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = 2
    a.record(stream)
    for _ in range(n):
        plan.run(stream=stream)
    b.record(stream)
    torch.cuda.synchronize()
    batch_ms = a.elapsed_time(b) / n
    ref = out.clone()

    def plain():
        for i, (k, r, dd, nd, vv, nn) in enumerate(tasks):
            ctxs[k].pe(out[i], rotation=r, det_begin=dd, det_count=nd, vox_begin=vv, vox_count=nn,
                       stream=stream)

    plain()                                                   # warm-up
    torch.cuda.synchronize()
    a.record(stream)
    plain()
    b.record(stream)
    torch.cuda.synchronize()
    plain_ms = a.elapsed_time(b)
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


# ---------------------------------------------------------------------------------------
# CPU baseline: the oracle (reference float arithmetic in C) on the host cores

def cpu_baseline(args, g, n_planes, budget_s=12.0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    plane = n_planes // 2 if n_planes > 1 else 0
    gp = plane_geometry(g, plane) if n_planes > 1 else g
    rng = np.random.default_rng(0)
    # detector rows sampled across the array, all voxels of the plane's middle rows
    nx = int(g.image[0])
    ny = int(g.image[1])
    v0 = nx * (ny // 2)
    nv = nx
    n_rows = 4
    # the FP64 oracle loop is the baseline; the FP32 twin (the reference's float arithmetic)
    # is timed on the same rows beside it
    while True:
        rows = np.sort(rng.choice(g.n_det, n_rows, replace=False))
        t = time.perf_counter()
        oracle.pe(gp, prec=64, dets=rows, v0=v0, nv=nv, threads=threads)
        dt = time.perf_counter() - t
        if dt > budget_s * 0.25 or n_rows >= g.n_det:
            break
        n_rows = min(g.n_det, int(n_rows * max(2.0, 0.6 * budget_s / max(dt, 1e-3))))
    t = time.perf_counter()
    oracle.pe(gp, prec=32, dets=rows, v0=v0, nv=nv, threads=threads)
    dt32 = time.perf_counter() - t
    el = n_rows * nv
    return {"value": el / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "fp32_twin_value": el / dt32,
            "sample": f"{n_rows} random crystals x {nv} voxels (one voxel row of z-plane {plane}); "
                      f"FP64 oracle, OpenMP, {dt:.1f} s (FP32 twin on the same rows: {dt32:.1f} s)"}


# ---------------------------------------------------------------------------------------
# reference arm: the reference's own CUDA program through its own host entry point

def run_reference(args, rank, world, local):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_lib
    g, n_planes, desc = workload(args.workload)
    if rank != 0:
        return None
    if not ref_lib.available():
        return {"impl": "reference", "unavailable": "oracle/_ref not built (make -C oracle ref)"}
    plane = n_planes // 2 if n_planes > 1 else 0
    ny = int(g.image[1])
    strip = args.ref_rows
    samples = []
    for k in range(args.warmup + args.steps):
        iy0 = (k * strip) % ny
        gs = geometry.voxel_slab(g, plane, iy0, strip) if n_planes > 1 else g
        samples.append(gs)
    for k in range(args.warmup):
        ref_lib.pe(samples[k], cuda_id=local)
    t = time.perf_counter()
    for k in range(args.warmup, args.warmup + args.steps):
        ref_lib.pe(samples[k], cuda_id=local)
    dt = time.perf_counter() - t
    nel = samples[0].n_det * samples[0].n_vox
    value = nel * args.steps / dt
    sample = (f"{strip} voxel rows x {int(g.image[0])} of z-plane {plane} x {g.n_det} crystals "
              f"({nel} elements) per step, one PESysMatGen call each")
    scatter = None if args.no_scatter else run_reference_scatter(ref_lib, local)
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded geometry)",
            "config": {"workload": desc, "sample": sample,
                       "build": "reference sources compiled for sm_100a (nvcc -O3, oracle/Makefile)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": sample + "; the reference is a CUDA program: its host "
                                       "wrapper drives the GPU"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": args.steps, "scatter": scatter}


def run_reference_scatter(ref_lib, local):
    """The reference's combined scatter program on 8 voxel rows (384 voxels) of configuration
    3's z-plane 8 x 1024 crystals: a warm-up call computes and writes the relationship bitmaps,
    the timed call reads them back (about 200 MB of files), as a rotation loop of the reference
    program would."""
    import tempfile
    g = geometry.voxel_slab(geometry.config3(), 8, 20, 8)
    pe = ref_lib.pe(g, cuda_id=local)
    tmp = tempfile.mkdtemp(prefix="refscatter_")
    ref_lib.scatter(g, pe, "combined", cuda_id=local, workdir=tmp)
    t = time.perf_counter()
    ref_lib.scatter(g, pe, "combined", cuda_id=local, workdir=tmp, load_bitmaps=True)
    dt = time.perf_counter() - t
    for f in os.listdir(tmp):
        os.remove(os.path.join(tmp, f))
    os.rmdir(tmp)
    nel = g.n_det * g.n_vox
    return {"value": nel / dt, "unit": UNIT, "ms_per_step": dt * 1e3,
            "workload": "config3 primary Compton (crystal + collimator), reference combined program, "
                        f"voxel rows 20-27 of z-plane 8: {g.n_det} crystals x {g.n_vox} voxels, bitmaps read "
                        "from the files of a warm-up call"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sysmat", choices=("sysmat", "reference"))
    ap.add_argument("--workload", default="config2", choices=("config1", "config2", "config3"))
    ap.add_argument("--ref-rows", type=int, default=4, help="voxel rows per reference step")
    ap.add_argument("--det-count", type=int, default=None,
                    help="first N crystals only (small cases for profiling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-scatter", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-sampled", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
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
            res = run_sysmat(args, rank, world, local)
            if rank == 0 and not args.no_cpu_baseline:
                g, n_planes, _ = workload(args.workload)
                res["cpu_baseline"] = cpu_baseline(args, g, n_planes)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
