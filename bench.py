"""Throughput benchmark of the FDTD timestep hot path on B200.

Workload: the two-sphere dielectric scene at 512^3 (spheres eps 4.0 r=80 at
(160,256,256) and eps 2.25 r=60 at (352,256,256)), 16-cell CPML, Gaussian Ez
source at (256,256,64), 8 Ez DFT probes on a line at z=448, FP32 fields.
A step is one full Yee timestep of the whole grid (H, E, CPML psi, source,
probes).  Metric: Mcell-updates/s = cells * steps / seconds / 1e6.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload two_spheres|random_spheres|demo_sphere|batched|closure]
                  [--grid N] [--precision f32|f16|bf16] [--scenes N]

--workload random_spheres --precision f16|bf16 measures the mixed-precision
form (32 seeded random spheres, sinusoid source, 16-cell CPML; fields stored
as 16-bit values with per-slab power-of-two scales, FP32 arithmetic) against
the same scene in FP32 (--precision f32).

Our arm prints one JSON line with `value` (device-resident, CUDA events on
the handle's stream), `e2e` (through the C ABI from host buffers: upload of
the scene, K steps, download of probe sums and one snapshot), `roofline`
(fused kernel: algorithmic bytes per launch / event-timed launch duration),
`cpu_baseline` (the CPU oracle restating the reference, timed on this host),
and `clocks` sampled by nvidia-smi during the timed region.  With N > 1
ranks (torchrun) the grid is split into one z slab per rank with 8-plane
ghost blocks exchanged every 8 steps over NCCL (strong scaling; the value
counts the whole grid's cells once); --replicas runs an independent copy of
the workload per rank instead (weak scaling, no collective).
The reference arm times the reference's CPU algorithm (the oracle port; the
Rust reference cannot be built here) with all host threads.
"""
from __future__ import annotations

import argparse
import copy
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-updates/s"
GRID = 512  # set by --grid (smaller grids are for profiling captures only)
N_CELLS = GRID ** 3
WORKLOAD = f"two_spheres_{GRID}^3_fp32_cpml16_gaussian_8probes"


PRECISION = "f32"
ELEM = {"f32": 4, "f16": 2, "bf16": 2}


def algorithmic_bytes(sc) -> int:
    """Per step (one launch of each fused work class): 6 fields read + written
    at the storage width plus 1 B material id per cell (49 B in FP32, 25 B in
    16-bit storage), plus 32 B per (cell, axis) inside that axis's graded
    slab (4 FP32 psi values read + written)."""
    n = (sc.dims.nx, sc.dims.ny, sc.dims.nz)
    cells = sc.dims.voxel_count()
    b = (12 * ELEM[PRECISION] + 1) * cells
    for ax in range(3):
        t = sc.pml.thickness_voxels[ax] if sc.pml else 0
        if t:
            b += 32 * (cells // n[ax]) * min(2 * t, n[ax])
    return b


def whole_job_value(world: int, cells: int, steps: int, seconds: float) -> float:
    """Mcell-updates/s of the whole job: every rank's cells over the slowest
    rank's time (ranks are replicas, so the work is world x cells x steps)."""
    return world * cells * steps / seconds / 1e6


def max_over_ranks(dist, value: float, device: str = "cuda") -> float:
    """The largest value over all ranks (the slowest rank's time); every rank
    calls it at the same point.  dist is torch.distributed or None (1 rank)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ms_so_far(e0, e1) -> float:
    """Seconds between two recorded, completed CUDA events."""
    return e0.elapsed_time(e1) / 1e3


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region
    (every 50 ms)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(", ") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(desc, seconds=15.0, seconds_one_core=6.0):
    """The oracle (C restatement of the reference, AVX2 rows, one worker
    thread per host core splitting each phase into contiguous block ranges
    like the reference's rayon Z-slabs) on a bounded sample: as many full
    steps of the workload as fit in about `seconds`; then the same on one
    core for about `seconds_one_core`.  The oracle builds the workload from
    its description with its own voxelizer and tables."""
    from oracle import oracle as O
    nt = os.cpu_count() or 1
    sim = O.sim_from_description(desc, steps=128)

    def timed(threads, budget):
        t0 = time.perf_counter()
        n = 0
        while n < 64:
            sim.step(1, threads)
            n += 1
            if time.perf_counter() - t0 > budget:
                break
        return n, time.perf_counter() - t0

    sim.step(1, nt)  # warm-up (page-in)
    n, el = timed(nt, seconds)
    n1, el1 = timed(1, seconds_one_core)
    sim.close()
    nx, ny, nz = desc["dims"]
    cells = nx * ny * nz
    return {"value": round(cells * n / el / 1e6, 2), "unit": METRIC, "cores": nt,
            "kind": "port", "sample": f"{n} full {GRID}^3 steps after 1 warm-up step, {el:.1f} s",
            "one_core": {"value": round(cells * n1 / el1 / 1e6, 2), "unit": METRIC,
                         "sample": f"the next {n1} steps on 1 thread, {el1:.1f} s"}}


def description(args, steps):
    """The workload as plain data (scene text, grid, dt/dx, CPML request,
    sources, probes): building it loads no library, so the reference arm
    can hand it to the oracle alone."""
    from wavefront_b200 import configs
    if args.workload == "random_spheres":
        return configs.random_spheres_desc(n=GRID, steps=steps)
    if args.workload == "demo_sphere":
        return configs.demo_sphere_cube_desc(n=GRID, steps=steps)
    return configs.two_spheres_desc(n=GRID, steps=steps)


def scenario(args, steps, device_voxelize=None):
    """The workload for the CUDA path; random spheres above 256^3 are
    voxelized on the device (the host voxelizer's 32 full-grid passes take
    minutes at 1024^3).  device_voxelize True leaves any text scene to the
    device voxelizer (the end-to-end leg: the scene text crosses the host
    link, not the ids)."""
    from wavefront_b200 import configs
    if device_voxelize is None:
        dv = args.workload == "random_spheres" and GRID > 256
    else:
        dv = bool(device_voxelize)
    return configs.from_desc(description(args, steps), device_voxelize=dv)


def scene_config(desc, precision=None) -> dict:
    """The workload keys both arms report (the reference arm stores FP32)."""
    p = precision or PRECISION
    return {"workload": WORKLOAD, "grid": [GRID] * 3,
            "cpml_cells": desc["pml"]["cells"] if desc["pml"] is not None else 0,
            "probes": len(desc["probes"]), "storage": p,
            "l2": f"inputs larger than L2 ({N_CELLS * 6 * ELEM[p] / 1e9:.1f} GB of fields "
                  "per state buffer)"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    # the oracle builds the workload from its plain description with its own
    # voxelizer and tables: this process never loads the CUDA library
    desc = description(args, args.warmup + args.steps)
    from oracle import oracle as O
    nt = os.cpu_count() or 1
    sim = O.sim_from_description(desc, steps=args.warmup + args.steps)
    budget = float(os.environ.get("WF_REF_SECONDS", "120"))
    for _ in range(args.warmup):
        sim.step(1, nt)
    t0 = time.perf_counter()
    n = 0
    while n < args.steps:
        sim.step(1, nt)
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    sim.close()
    v = N_CELLS * n / el / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": METRIC,
        "n_gpus": world, "steps": n, "warmup": args.warmup, "ms_per_step": round(el / n * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": scene_config(desc, "f32"),
        "cpu_baseline": {"value": round(v, 2), "unit": METRIC, "cores": nt, "kind": "port",
                         "sample": f"{n} of {args.steps} requested {GRID}^3 steps in {el:.1f} s "
                                   "(time-bounded); the Rust reference cannot be built here, so "
                                   "this is the oracle's C restatement of its f32 AVX2 path"},
        "e2e": {"value": round(v, 2), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_batched(args, rank, world, local_rank):
    """Batched sweep: 256 independent cubes (edges 32..128, 1-4 primitives,
    exact 10-cell CPML, Ricker source, one probe each; --scenes takes the first
    N of them, for a small profiling case) stepped together by one persistent
    launch per CPML class per step (wf_batch_step, 32-step graph replays),
    tiling from the batch autotuner.  value = total cells x steps / time."""
    import torch
    from wavefront_b200 import configs
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    total = args.warmup + args.steps
    scenes = configs.batched_sweep(256, steps=total)[:args.scenes]
    cells = sum(sc.dims.voxel_count() for sc in scenes)
    b = configs.device_batch(scenes, device=local_rank)
    if args.tiling:
        b.set_tiling(*[int(v) for v in args.tiling.split(",")])
        tuned_ms = None
    else:
        _, tuned_ms = b.autotune(2)
    tiling = b.tiling()
    b.step(args.warmup)
    b.sync()
    stream = torch.cuda.ExternalStream(b.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    k0 = b.kernel_launches
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        b.step(args.steps)
        e1.record(stream)
        b.sync()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = b.kernel_launches - k0
    b.close()
    ms = max_over_ranks(dist, ms)
    value = whole_job_value(world, cells, args.steps, ms / 1e3)
    alg = sum(algorithmic_bytes(sc) for sc in scenes)
    achieved = alg / (ms / args.steps / 1e3) / 1e9
    peak, peak_kind = peaks()

    # end to end: upload every scene (ids, tables), step, read every probe's
    # sums; the batch's device allocation is set-up, outside the timed region
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    from wavefront_b200.engine import DeviceBatch
    b = DeviceBatch([sc.dims for sc in scenes], device=local_rank)
    b.sync()
    t0 = time.perf_counter()
    configs.load_batch(b, scenes)
    b.set_tiling(*tiling)
    b.sync()
    t_loaded = time.perf_counter()
    b.step(args.steps)
    b.sync()
    t_stepped = time.perf_counter()
    sums = [b.grid(i).probe_sums(0, 1) for i in range(len(scenes))]
    e2e_s = time.perf_counter() - t0
    phases = {"upload": round((t_loaded - t0) * 1e3, 1),
              "steps": round((t_stepped - t_loaded) * 1e3, 1),
              "probe_sums": round((t0 + e2e_s - t_stepped) * 1e3, 1)}
    b.close()
    e2e_s = max_over_ranks(dist, e2e_s)
    if dist:
        dist.barrier()
    e2e = whole_job_value(world, cells, args.steps, e2e_s)
    h2d = cells + len(scenes) * (256 * 16 + total * (4 + 8 * 2))
    d2h = len(sums) * 24

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "scenes": len(scenes), "cells_per_step": cells,
                       "edges": sorted({sc.dims.nx for sc in scenes}), "cpml_cells": 10,
                       "kernel": "persistent batched fused step + batched tail, CUDA graph",
                       "tiling": {"tile_rows": tiling[0], "z_chunk": tiling[1],
                                  "stages": tiling[2]},
                       "autotuned_ms_per_step": tuned_ms,
                       "l2": f"inputs larger than L2 ({cells * 24 / 1e9:.1f} GB of fields per "
                             "state buffer)",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "e2e": {"value": round(e2e, 1), "unit": METRIC,
                    "h2d_bytes_per_step": int(h2d / args.steps),
                    "d2h_bytes_per_step": int(d2h / args.steps),
                    "includes": "every scene's ids + tables uploaded, K steps, every probe's "
                                "sums read back; the batch's device allocation is untimed set-up",
                    "phases_ms": phases},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": None, "algorithmic_bytes_per_launch": alg,
                         "kernel_ms_per_launch": round(ms / args.steps, 4),
                         "launch": "one batched step (step kernel + tail)"},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline_batched(scenes)
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def cpu_baseline_batched(scenes, seconds=15.0):
    """The oracle on a bounded sample of the batch: scenes in order, 10 steps
    each, all host threads per scene, until about `seconds` have passed."""
    from oracle import oracle as O
    nt = os.cpu_count() or 1
    done = 0
    t0 = time.perf_counter()
    k = 0
    for sc in scenes:
        sim = O.sim_from_scenario(sc, steps=10)
        sim.step(10, nt)
        sim.close()
        done += sc.dims.voxel_count() * 10
        k += 1
        if time.perf_counter() - t0 > seconds:
            break
    el = time.perf_counter() - t0
    return {"value": round(done / el / 1e6, 2), "unit": METRIC, "cores": nt, "kind": "port",
            "sample": f"first {k} scenes x 10 steps each, {el:.1f} s (scene setup included)"}


def run_closure(args, rank, world, local_rank):
    """Learned thin-CPML closure: wall time of the same 224^3 physical
    interior with a 16-cell CPML (256^3 cells) and with the 4-cell thin layer
    (232^3 cells) alone and with the closure network applied every step (a
    Ricker Ez source at the centre, vacuum), plus the reflection test (48^3
    interior, 260 steps, against a reference domain nothing returns from)
    of a closure trained here on teacher-forced samples (96 runs of 64^3)."""
    import torch
    from wavefront_b200 import closure as CL
    from wavefront_b200 import configs
    from wavefront_b200.engine import DeviceFieldGrid
    from wavefront_b200.layout import GridDims, MaterialGrid, MaterialTable, PmlConfig, PmlContext
    from wavefront_b200.source import FieldComponent, Source, default_waveform
    torch.cuda.set_device(local_rank)
    if rank != 0:
        return
    interior = args.grid or 224
    dx = 1.0e-3
    dt = configs.courant_dt(dx)
    wf_ = default_waveform("ricker", float(np.float32(configs.C0 / (20.0 * dx))))
    total = args.warmup + args.steps
    if args.closure_timing_only:
        net = CL.ClosureNet(device=local_rank, seed=1)
    else:
        X, R, F, _ = CL.generate(96, seed=1, device=local_rank)
        net, _ = CL.train(X, R, F, 1.0, iters=4000, lr=3e-4, device=local_rank)
        del X, R, F

    def timed(n, pml, closure):
        dims = GridDims(n, n, n)
        g = DeviceFieldGrid(dims, kernel="fused", device=local_rank)
        try:
            g.set_materials(MaterialGrid(dims), MaterialTable.vacuum_filled(dt, dx))
            if pml == "thin":
                CL.set_thin_cpml(g, dt, dx)
            else:
                g.set_pml(pml)
            c = n // 2
            s = Source(c, c, c, FieldComponent.Ez, 1.0, wf_)
            g.add_source_values(s.x, s.y, s.z, s.component, s.values(dt, total))
            if closure:
                net.attach(g, 0.5)
            g.step(args.warmup)
            g.sync()
            st = torch.cuda.ExternalStream(g.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            k0 = g.kernel_launches
            e0.record(st)
            g.step(args.steps)
            e1.record(st)
            g.sync()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / args.steps, g.kernel_launches - k0
        finally:
            g.close()

    n16 = interior + 32
    thick_ms, _ = timed(n16, PmlContext.build(GridDims(n16, n16, n16), PmlConfig(thickness=16), dt, dx),
                        False)
    with ClockSampler(local_rank) as clk:
        closure_ms, launches = timed(interior + 8, "thin", True)
    thin_ms, _ = timed(interior + 8, "thin", False)
    refl = {} if args.closure_timing_only else {
        k: CL.reflection_test(**kw)["max_rel_error"] for k, kw in (
            ("thin_layer_alone", {"truncated": True}),
            ("thin_layer_with_closure_gain_0.5", {"net": net, "alpha": 0.5, "truncated": True}),
            ("thin_layer_with_closure_gain_1_energy_guard",
             {"net": net, "alpha": 1.0, "truncated": True, "guard": True}),
            ("thin_layer_with_closure_gain_0.5_energy_guard",
             {"net": net, "alpha": 0.5, "truncated": True, "guard": True}),
            ("plain_cpml_4", {"cpml": 4}), ("plain_cpml_16", {"cpml": 16}))}
    value = interior ** 3 / (closure_ms / 1e3) / 1e6
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(closure_ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "interior": [interior] * 3,
                   "cells_counted": f"physical interior ({interior}^3) per step",
                   "closure": "per-face 3x3x3 conv 10-16-16-6, GELU, bf16 weights, fp32 accumulation, "
                              "8-cell band, correction gain 0.5",
                   "parallelism": "1 GPU"},
        "comparison_ms_per_step": {f"cpml16_{n16}^3": round(thick_ms, 4),
                                   f"thin4_{interior + 8}^3_with_closure": round(closure_ms, 4),
                                   f"thin4_{interior + 8}^3_alone": round(thin_ms, 4)},
        "reflection_test_max_rel_error": {k: (round(v, 5) if np.isfinite(v) else None)
                                          for k, v in refl.items()},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_conv(args, rank, world, local_rank):
    """The closure network's convolutions alone, at the closure's size (6 face
    bands of 8 x 232 x 232 voxels, --grid sets the band's edge): one forward
    convolution with GELU per layer shape (10->16, 16->16, 16->6), on the
    tensor cores (tcgen05 implicit GEMM) and on the CUDA cores; CUDA events
    over `--steps` launches after `--warmup`.  value = useful TFLOP/s of the
    16->16 layer on the tensor cores."""
    import ctypes as C

    import torch
    from wavefront_b200 import _lib as L
    torch.cuda.set_device(local_rank)
    if rank != 0:
        return
    n, D, H = 6, 8, args.grid or 232
    dev = torch.device("cuda", local_rank)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    out, launches = {}, 0
    face = torch.arange(6, dtype=torch.int32, device=dev)
    gen = torch.Generator(device=dev).manual_seed(0)
    with ClockSampler(local_rank) as clk:
        for ci, co in ((10, 16), (16, 16), (16, 6)):
            x = torch.randn(n, ci, D, H, H, device=dev, generator=gen)
            wb = (torch.randn(6, co, ci, 27, device=dev, generator=gen) * 0.2).to(torch.bfloat16)
            z = torch.empty(n, co, D, H, H, device=dev)
            a = torch.empty_like(z)
            for tc in (1, 0):
                L.lib().wf_nn_set_tensor_cores(tc)

                def conv():
                    L.check(L.lib().wf_nn_conv3d_forward(
                        C.c_void_p(x.data_ptr()), C.c_void_p(wb.data_ptr()),
                        C.c_void_p(face.data_ptr()), C.c_void_p(z.data_ptr()),
                        C.c_void_p(a.data_ptr()), n, ci, co, D, H, H, 1, st))
                for _ in range(args.warmup):
                    conv()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(args.steps):
                    conv()
                e1.record()
                torch.cuda.synchronize()
                launches += args.steps
                ms = e0.elapsed_time(e1) / args.steps
                flops = 2.0 * n * D * H * H * ci * co * 27
                out[f"{ci}->{co}_{'tensor_cores' if tc else 'cuda_cores'}"] = {
                    "ms": round(ms, 4), "tflops": round(flops / ms / 1e9, 1)}
    L.lib().wf_nn_set_tensor_cores(1)
    v = out["16->16_tensor_cores"]["tflops"]
    print(json.dumps({
        "metric": "closure conv TFLOP/s (useful, 16->16 layer, tensor cores)", "value": v,
        "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": out["16->16_tensor_cores"]["ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 x3 parts, fp32 accumulate",
        "data": "synthetic",
        "config": {"workload": f"closure_conv_6_faces_8x{H}x{H}", "layers": out,
                   "parallelism": "1 GPU"},
        "e2e": {"value": None, "unit": "TFLOP/s", "skipped": "a kernel micro-benchmark"},
        "gpu_launches": launches, "clocks": clk.summary()}), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    from wavefront_b200 import configs
    from wavefront_b200.engine import DeviceFieldGrid
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    total = args.warmup + args.steps
    desc = description(args, total)
    sc = scenario(args, total)

    def load(g, extra=0, sc=sc):
        """Scene or material ids, CPML profiles, tiling, source values and probe
        tables (for the run's steps plus `extra`) into a fresh handle."""
        if sc.grid is None:  # the device voxelizer registers the scene's materials
            g.set_scene(sc.scene_text, copy.deepcopy(sc.table), sc.dt, sc.dx)
        else:
            g.set_materials(sc.grid, sc.table)
        if sc.pml is not None:
            g.set_pml(sc.pml)
        if args.tiling:
            g.set_tiling(*[int(v) for v in args.tiling.split(",")])
        if args.columns == "off":
            g.set_column_tiles(False)
        for s in sc.sources:
            g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, total + extra))
        for p in sc.probes:
            c, si = p.tables(sc.dt, total + extra)
            g.add_probe_tables(p.x, p.y, p.z, p.component, c, si, p.first_step(sc.dt))
        return g

    # the value leg's handle has tables for EXTRA more steps: the untimed steps
    # that keep the clock sampler busy after the timed region
    EXTRA = 640

    def build(kernel="fused"):
        return load(DeviceFieldGrid(sc.dims, kernel=kernel, device=local_rank, precision=PRECISION),
                    EXTRA)

    # ---- device-resident throughput (value) + fused-kernel roofline -------
    tcold = time.perf_counter()
    g = build()
    if PRECISION == "f32" and not args.no_e2e:
        g.reserve_download()  # the e2e leg's snapshot staging buffer, cached when g closes
    g.sync()
    cold_create_ms = (time.perf_counter() - tcold) * 1e3
    tiling = list(g.tiling())
    column_tiles = g.column_tiles
    g.step(args.warmup)
    g.sync()
    g.set_timing(True)
    stream = torch.cuda.ExternalStream(g.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    k_before = g.kernel_launches
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        g.step(args.steps)
        e1.record(stream)
        g.sync()
        torch.cuda.synchronize()
        gpu_launches = g.kernel_launches - k_before
        kern_ms, launches = g.timing()
        g.set_timing(False)
        # a short timed region holds at most a sample or two at the sampler's
        # rate: keep the same kernels running (untimed) for about half a second
        # so that the clock record has samples under the same load
        t_extra, extra = time.perf_counter(), 0
        while time.perf_counter() - t_extra < 0.5 - ms_so_far(e0, e1) and extra + 32 <= EXTRA:
            g.step(32)
            g.sync()
            extra += 32
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    g.set_timing(False)
    g.close()
    clocks = clk.summary()
    ms = max_over_ranks(dist, ms)
    value = whole_job_value(world, N_CELLS, args.steps, ms / 1e3)

    alg = algorithmic_bytes(sc)
    per_launch_ms = kern_ms / max(launches, 1)
    achieved = alg / (per_launch_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf) and args.workload == "two_spheres" and GRID == 512 and PRECISION == "f32":
        with open(tf) as f:
            traffic = json.load(f).get("fused_two_spheres_512_bytes_per_launch")

    # ---- end to end through the C ABI from host buffers -----------------
    e2e_line = {"value": None, "unit": METRIC, "skipped": "--no-e2e"}
    if not args.no_e2e:
        # a text scene is voxelized on the device (its ids equal the host
        # voxelizer's), so the scene text crosses the host link, not the ids;
        # host ids travel pinned
        sce = scenario(args, total, device_voxelize=True) if (desc["scene"] or {}).get("text") else sc
        if sce.grid is not None:
            pin_ids = torch.from_numpy(sce.grid.ids).pin_memory()
        snap = torch.empty(N_CELLS * 6, dtype=torch.float32).pin_memory()
        if sce.grid is not None:
            sce.grid.ids = pin_ids.numpy()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

        def e2e_run(snapshot: bool):
            """Seconds for one run through the C ABI, everything timed (the
            handle's creation too: its device memory comes from the library's
            cache of the blocks the first handle freed), and the phases."""
            t0 = time.perf_counter()
            g = DeviceFieldGrid(sc.dims, kernel="fused", device=local_rank, precision=PRECISION)
            async_snap = snapshot and PRECISION == "f32"
            if async_snap:
                g.reserve_download()  # the snapshot's staging buffer
            tc = time.perf_counter()
            load(g, sc=sce)
            g.sync()
            t_built = time.perf_counter()
            # with `snapshot`, the FieldBlock snapshot of step 0, as the
            # reference's benchmark writes one (--snapshot-every beyond the step
            # count): FP32 storage downloads it while the other steps run, like
            # the reference's double-buffered writer, 16-bit storage after them
            g.step(1)
            if async_snap:
                g.download_blocks_async(snap.numpy())
            g.step(args.steps - 1)
            sums = [g.probe_sums(i, 1) for i in range(len(sc.probes))]
            t_stepped = time.perf_counter()
            if snapshot and not async_snap:
                import ctypes as C
                from wavefront_b200 import _lib as L
                L.check(L.lib().wf_download_blocks(g._h, C.c_void_p(snap.data_ptr())), g._h)
            g.sync()
            el = time.perf_counter() - t0
            phases = {"create": round((tc - t0) * 1e3, 1), "upload": round((t_built - tc) * 1e3, 1),
                      "steps_and_probe_sums": round((t_stepped - t_built) * 1e3, 1)}
            if snapshot:
                phases["snapshot_wait"] = round((t0 + el - t_stepped) * 1e3, 1)
            g.close()
            return el, phases, len(sums)

        e2e_s, phases, nsums = e2e_run(False)
        phases["first_handle_create_and_upload_cold_untimed"] = round(cold_create_ms, 1)
        snap_s, snap_phases, _ = e2e_run(True)
        e2e_s = max_over_ranks(dist, e2e_s)
        snap_s = max_over_ranks(dist, snap_s)
        if dist:
            dist.barrier()
        e2e = whole_job_value(world, N_CELLS, args.steps, e2e_s)
        h2d = (N_CELLS if sce.grid is not None else len(sce.scene_text)) + 256 * 16 + total * (4 + 8 * 16)
        d2h = nsums * (8 * 2 + 8)
        e2e_line = {"value": round(e2e, 1), "unit": METRIC,
                    "h2d_bytes_per_step": int(h2d / args.steps),
                    "d2h_bytes_per_step": int(d2h / args.steps),
                    "includes": "the handle's creation (device memory from the library's "
                                "cache, warmed by the first handle of the run), the scene text "
                                "voxelized on the device (or material ids uploaded pinned), CPML "
                                "and source/probe table uploads, K steps, "
                                "every probe's DFT sums read back (the run's result)",
                    "phases_ms": phases,
                    "with_snapshot": {
                        "value": round(whole_job_value(world, N_CELLS, args.steps, snap_s), 1),
                        "d2h_bytes_per_step": int((d2h + N_CELLS * 24) / args.steps),
                        "includes": "the same plus the FieldBlock snapshot of step 0 (3.2 GB at "
                                    "512^3) downloaded to pinned memory, FP32 while the other "
                                    "steps run; bound by the host link at 20 steps",
                        "phases_ms": snap_phases}}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {**scene_config(desc), "kernel": "fused TMA z-march", "arith": "exact (no FMA)",
                       "x_cpml_column_tiles": column_tiles,
                       "tiling": {"tile_rows": tiling[0], "z_chunk": tiling[1],
                                  "stages": tiling[2]},
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "e2e": e2e_line,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": traffic, "algorithmic_bytes_per_launch": alg,
                         "kernel_ms_per_launch": round(per_launch_ms, 4)},
            "gpu_launches": int(gpu_launches),
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu and sc.grid is not None:
            line["cpu_baseline"] = cpu_baseline(desc)
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_slabs(args, local_rank):
    """The workload split into `--slabs` z slabs on one GPU (SlabDomain: one
    handle per slab on a stream of its own, 8-plane ghost blocks refreshed
    every 8 steps by the pack/unpack kernels).  value counts the whole grid's
    cells once; the ghost planes are the decomposition's extra work."""
    import torch
    from wavefront_b200 import slabs as S
    torch.cuda.set_device(local_rank)
    total = args.warmup + args.steps
    desc = description(args, total)
    sc = scenario(args, total)
    d = S.SlabDomain(sc, args.slabs, steps=total, device=local_rank)
    if args.tiling:
        for st in d.states:
            st.grid.set_tiling(*[int(v) for v in args.tiling.split(",")])
    d.step(args.warmup)
    d.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k_before = sum(st.grid.kernel_launches for st in d.states)
    x_before = d.exchanges
    with ClockSampler(local_rank) as clk:
        e0.record(d.stream)
        d.step(args.steps)
        e1.record(d.stream)
        d.sync()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    # each exchange: two packs and two unpacks per neighbouring pair
    launches = (sum(st.grid.kernel_launches for st in d.states) - k_before
                + 4 * (args.slabs - 1) * (d.exchanges - x_before))
    planes = sum(s.nz for s in d.slabs)
    d.close()
    value = whole_job_value(1, N_CELLS, args.steps, ms / 1e3)
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {**scene_config(desc), "slabs": args.slabs, "ghost_planes": S.GHOST,
                   "exchange_every_steps": S.GHOST, "planes_stepped_per_step": planes,
                   "parallelism": f"z slabs x{args.slabs} on 1 GPU"},
        "e2e": {"value": None, "unit": METRIC, "skipped": "--slabs measures the decomposition"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_slab_ranks(args, rank, world, local_rank, make_state=None):
    """The workload split into one z slab per rank (SlabRank): each rank
    steps its slab and exchanges 8-plane ghost blocks with its neighbours
    every 8 steps (NCCL by default; --backend gloo stages them through pinned
    host buffers).  Strong scaling: the whole grid is fixed, value counts its
    cells once over the slowest rank's time.  make_state replaces the device
    slab (a CPU test drives this leg with oracle slabs over gloo; times are
    then host clocks)."""
    import datetime

    import torch
    import torch.distributed as dist
    from wavefront_b200 import slabs as S
    gpu = make_state is None
    dev = 0
    if gpu:
        dev = local_rank % torch.cuda.device_count()
        torch.cuda.set_device(dev)
    dist.init_process_group(args.backend, timeout=datetime.timedelta(seconds=300))
    red = "cuda" if gpu and args.backend == "nccl" else "cpu"
    try:
        total = args.warmup + args.steps
        desc = description(args, total)
        sc = scenario(args, total)

        def drain(r):
            if r.stream is not None:
                r.stream.synchronize()

        r = S.SlabRank(sc, steps=total, make_state=make_state)
        if args.tiling and gpu:
            r.state.grid.set_tiling(*[int(v) for v in args.tiling.split(",")])
        r.step(args.warmup)
        drain(r)
        k_before = r.state.grid.kernel_launches if gpu else 0
        x_before = r.exchanges
        dist.barrier()
        if gpu:
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev) as clk:
            if gpu:
                e0.record(r.stream)
            t0 = time.perf_counter()
            r.step(args.steps)
            drain(r)
            wall_ms = (time.perf_counter() - t0) * 1e3
            if gpu:
                e1.record(r.stream)
                r.stream.synchronize()
                torch.cuda.synchronize()
        dist.barrier()
        ms = max_over_ranks(dist, e0.elapsed_time(e1) if gpu else wall_ms, device=red)
        # this rank's step kernels plus its packs and unpacks (one each per neighbour)
        nbrs = (rank > 0) + (rank < world - 1)
        launches = ((r.state.grid.kernel_launches - k_before) if gpu else 0) + \
            2 * nbrs * (r.exchanges - x_before)
        planes = r.slab.nz
        r.close()
        value = whole_job_value(1, N_CELLS, args.steps, ms / 1e3)

        # end to end from host buffers: every rank builds its slab (allocation,
        # ids, tables), steps, and the probe sums are gathered on rank 0
        dist.barrier()
        t0 = time.perf_counter()
        r = S.SlabRank(sc, steps=total, make_state=make_state)
        r.step(args.steps)
        drain(r)
        sums = r.gather_probe_sums(1)
        e2e_s = max_over_ranks(dist, time.perf_counter() - t0, device=red)
        r.close()
        e2e = whole_job_value(1, N_CELLS, args.steps, e2e_s)
        if rank == 0:
            gpus = min(world, torch.cuda.device_count()) if gpu else 0  # ranks may share a GPU
            h2d = N_CELLS + 256 * 16 + total * (4 + 8 * 16)
            line = {
                "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": gpus,
                "ranks": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {**scene_config(desc), "slabs": world, "ghost_planes": S.GHOST,
                           "exchange_every_steps": S.GHOST,
                           "rank0_planes_stepped_per_step": planes,
                           "parallelism": f"z slabs x{world}, {args.backend} exchange"},
                "e2e": {"value": round(e2e, 1), "unit": METRIC,
                        "h2d_bytes_per_step": int(h2d / args.steps),
                        "d2h_bytes_per_step": int(len(sums or {}) * 24 / args.steps),
                        "includes": "every rank's slab set-up (handle allocation, ids, CPML and "
                                    "source/probe tables), K steps with ghost-block exchanges, "
                                    "probe sums gathered on rank 0"},
                "gpu_launches": int(launches),
                "clocks": clk.summary(),
            }
            print(json.dumps(line), flush=True)
    finally:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--tiling", default="", help="tile_rows,z_chunk,stages")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end leg (its snapshot needs 24 B/cell of pinned host RAM)")
    ap.add_argument("--grid", type=int, default=0,
                    help="cube edge (default 512 for two_spheres, 1024 for random_spheres)")
    ap.add_argument("--workload", default="two_spheres",
                    choices=["two_spheres", "random_spheres", "batched", "closure", "conv",
                             "demo_sphere"],
                    help="two_spheres: the 512^3 headline; random_spheres: the mixed-precision "
                         "scene; demo_sphere: the reference's own benchmark shape (256^3 demo "
                         "sphere, 8-cell CPML)")
    ap.add_argument("--scenes", type=int, default=256,
                    help="batched workload: use the first N of its 256 scenes (profiling)")
    ap.add_argument("--slabs", type=int, default=0,
                    help="two_spheres/random_spheres/demo_sphere on one GPU split into this many "
                         "z slabs with ghost-block exchange (FP32)")
    ap.add_argument("--columns", default="on", choices=["on", "off"],
                    help="x-CPML slabs as 16-wide column tiles (on) or inside the wide tiles")
    ap.add_argument("--closure-timing-only", action="store_true",
                    help="closure workload: untrained random weights, no training and no "
                         "reflection test (wall times only; for profiling)")
    ap.add_argument("--replicas", action="store_true",
                    help="under torchrun: an independent replica of the workload per rank "
                         "(weak scaling) instead of one z slab per rank")
    ap.add_argument("--backend", default="nccl", choices=["nccl", "gloo"],
                    help="--slabs under torchrun: how ghost blocks travel between ranks")
    ap.add_argument("--precision", default="f32", choices=["f32", "f16", "bf16"],
                    help="field storage (16-bit: per-slab power-of-two scales, FP32 math)")
    args = ap.parse_args()
    global GRID, N_CELLS, WORKLOAD, PRECISION
    GRID = args.grid or {"random_spheres": 1024, "demo_sphere": 256}.get(args.workload, 512)
    N_CELLS = GRID ** 3
    PRECISION = args.precision
    if args.workload == "batched":
        WORKLOAD = "batched_sweep_256_scenes_32-128^3_fp32_cpml10_ricker"
    elif args.workload == "closure":
        WORKLOAD = f"learned_closure_{args.grid or 224}^3_interior_thin4_vs_cpml16_ricker"
    elif args.workload == "random_spheres":
        WORKLOAD = f"random_spheres_{GRID}^3_{PRECISION}_storage_cpml16_sinusoid_8probes"
    elif args.workload == "demo_sphere":
        WORKLOAD = f"demo_sphere_{GRID}^3_{PRECISION}_storage_cpml8_ricker"
    elif PRECISION == "f32":
        WORKLOAD = f"two_spheres_{GRID}^3_fp32_cpml16_gaussian_8probes"
    else:
        WORKLOAD = f"two_spheres_{GRID}^3_{PRECISION}_storage_cpml16_gaussian_8probes"
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.gpus == 1 else 1)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "batched":
        run_batched(args, rank, world, local_rank)
    elif args.workload == "closure":
        run_closure(args, rank, world, local_rank)
    elif args.workload == "conv":
        run_conv(args, rank, world, local_rank)
    elif args.slabs or (world > 1 and not args.replicas and PRECISION == "f32"):
        # under torchrun the grid is split into one z slab per rank (strong
        # scaling); --replicas runs an independent copy per rank instead
        if PRECISION != "f32":
            raise SystemExit("--slabs needs FP32 storage")
        if world > 1:
            if args.slabs and args.slabs != world:
                raise SystemExit("under torchrun --slabs must equal the number of ranks")
            run_slab_ranks(args, rank, world, local_rank)
        else:
            run_slabs(args, local_rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
