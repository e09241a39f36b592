"""Benchmark of the UniformCUDA projection: MAC cells projected per second at a 1e-6 residual.

Workload (one step): a 2048 x 2048 two-phase dam break (liquid 1000 / gas 1, liquid below half
height plus a seeded 200x300 block, face velocities U[-1, 1] in FP32), gravity -9.8 applied,
then one pressure projection: coefficients and multigrid rebuilt from the step's masses, MG-PCG
to the reference's own stop rule (max |r| <= 1e-6 dx^2/dt on the FP64 residual,
FluidGridCPU.cpp:1093), velocity update, divergence check. The reference arm runs the same
scene, rule and config, so the two lines measure the same work. Inputs are seeded synthetic
data; the reference publishes no dataset for this path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

With N > 1 and no WORLD_SIZE in the environment the script starts itself under
torch.distributed.run, one rank per GPU, each projecting its own grid (independent replicas:
the path has no exchange step). Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "MAC cells projected/s at 1e-6 residual"
UNIT = "cells/s"
L2_FLUSH_BYTES = 256 << 20
# Algorithmic bytes per fine cell of the two fused fine-level smoothing kernels (FP32):
# pre reads r, right, down and the inverse diagonal and writes the pre-smoothed solution plus a
# quarter cell of coarse rhs; post reads the pre-smoothed solution, a quarter cell of coarse
# solution, r, right, down and the inverse diagonal and writes z.
ALGORITHMIC_BYTES = {0: 4 + 4 + 4 + 4 + 4 + 1, 1: 4 + 1 + 4 + 4 + 4 + 4 + 4}
KERNEL_NAMES = {0: "k_smooth_pre (fine level)", 1: "k_smooth_post (fine level)"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    p.add_argument("--size", type=int, default=2048)
    p.add_argument("--tolerance", type=float, default=1e-6)
    p.add_argument("--no-batched", action="store_true", help="skip the batched uneven-grid measurement")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-serve", action="store_true", help="skip the serving (continuous batching) measurement")
    p.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison")
    p.add_argument("--no-steps", action="store_true", help="skip the full-step (transport + projection) measurement")
    p.add_argument("--no-rules", action="store_true",
                   help="skip the relative-rule FP32 and reference-rule FP64 legs of the headline scene")
    p.add_argument("--no-viscous", action="store_true",
                   help="skip the 4096x4096 variable-viscosity comparison of FP32 and mixed precision")
    p.add_argument("--tail-cells", type=int, default=0,
                   help="multigrid tail threshold in cells (0: autotuned); pins the schedule for profiling")
    p.add_argument("--serve-requests", type=int, default=16)
    p.add_argument("--serve-steps", type=int, default=300)
    p.add_argument("--launch", choices=["graph", "stream"], default="graph",
                   help="stream: host-driven launches of the same kernels (for per-kernel profilers)")
    return p.parse_args()


def scene_for(size, rank):
    from fluidsim_b200 import scenes

    return scenes.dam_break(size, size, seed=1234 + rank, obstacles=0, velocity=1.0)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per fine cell of the fused smoothing kernels, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return {int(k): float(v) for k, v in json.load(f).get("dram_bytes_per_cell", {}).items()}


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device = device_index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"fluidsim_clocks_{os.getpid()}_rank{device_index}.csv")

    def __enter__(self):
        try:
            self.file = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.file.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# CPU legs (the reference engine compiled from its own sources, else the C restatement)
# ---------------------------------------------------------------------------------------------

def cpu_projection(scene, tolerance, threads, outputs=None):
    """Runs one step of the workload on the host; returns (seconds, iterations, kind). With an
    `outputs` dict and the reference engine available, its final u, v and p are stored there."""
    from oracle import oracle

    if oracle.reference_available():
        oracle.set_reference_threads(threads)
        g = oracle.ReferenceGrid(scene.width, scene.height, scene.cell_size, scene.liquid_density, scene.gas_density)
        g.set_gravity(scene.gravity)
        g.upload(scene.fraction, scene.u, scene.v, None, scene.liquid_mass[0], scene.gas_mass[0])
        t = time.perf_counter()
        g.apply_gravity(scene.dt)
        # The reference runs its own stop rule, max |div u| <= tol (FluidGridCPU.cpp:1093).
        r = g.project(scene.dt, 200, tolerance)
        seconds = time.perf_counter() - t
        if outputs is not None:
            _, outputs["u"], outputs["v"], outputs["p"] = g.download()
        return seconds, r.iterations, "reference"
    oracle.build(reference=False)
    g = oracle.OracleGrid(scene.width, scene.height, scene.cell_size)
    g.upload(scene.density(), scene.u, scene.v)
    t = time.perf_counter()
    g.apply_gravity(scene.gravity, scene.dt)
    r = g.project(scene.dt, 200, tolerance, relative_tolerance=tolerance)
    return time.perf_counter() - t, r.iterations, "port"


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


RULE = "reference: max |r| <= tolerance * dx^2 / dt on the FP64 residual (FluidGridCPU.cpp:1093)"


def workload_config(size, tolerance):
    """The `config` of both arms' lines: the same scene, stop rule and tolerance."""
    return {"workload": f"dam_break_{size}x{size} projection (gravity + MG-PCG to the reference's stop rule)",
            "cells": size * size, "tolerance": tolerance, "stop_rule": RULE, "density_ratio": "1000:1",
            "l2": "GPU: flushed (256 MiB write) before every timed step; host: inputs larger than L2"}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    size = args.size
    scene = scene_for(size, 0)
    threads = min(8, host_threads())
    times, iters, kind = [], [], "reference"
    for i in range(args.warmup + args.steps):
        seconds, it, kind = cpu_projection(scene, args.tolerance, threads)
        if i >= args.warmup:
            times.append(seconds)
            iters.append(it)
    per_step = statistics.mean(times)
    value = scene.cells / per_step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(size, args.tolerance),
        "iterations": statistics.mean(iters),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{args.steps} projections of the {size}x{size} workload, FluidGridCPU::project"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


# ---------------------------------------------------------------------------------------------
# CUDA arm
# ---------------------------------------------------------------------------------------------

class ProjectionTimer:
    """Times gravity + one projection of a scene from the same initial state every step: the
    state is copied back from a pristine grid, the L2 flushed, and the step timed with CUDA
    events on the grid's stream."""

    def __init__(self, scene, precision, torch, flush, tail_cells=0, tune=True):
        from fluidsim_b200 import FluidGrid, scenes

        self.scene, self.torch, self.flush = scene, torch, flush
        self.pristine = FluidGrid(scene.width, scene.height, scene.cell_size, precision)
        scenes.upload_scene(self.pristine, scene)
        self.work = FluidGrid(scene.width, scene.height, scene.cell_size, precision)
        self.work.configureMaterials([scene.liquid_density], [scene.gas_density])
        self.work.setGravityY(scene.gravity)
        self.work.copyStateFrom(self.pristine)
        self.tail_cells, self.vcycle_ms = tail_cells, None
        if tail_cells > 0:
            self.work.setTailCells(tail_cells)
        elif tune:
            # The multigrid schedule picked by the autotuner (timed V-cycles, outside the timed steps).
            self.tail_cells, self.vcycle_ms = self.work.autotune(10)
        self.stream = torch.cuda.ExternalStream(self.work.stream())

    def step(self, tolerance, relative):
        torch, scene = self.torch, self.scene
        self.work.copyStateFrom(self.pristine)
        with torch.cuda.stream(self.stream):
            self.flush.fill_(1.0)
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(self.stream)
        self.work.applyGravity(scene.dt)
        if relative:
            r = self.work.project(scene.dt, 400, tolerance, relative_tolerance=tolerance)
        else:
            r = self.work.project(scene.dt, 400, tolerance)
        stop.record(self.stream)
        stop.synchronize()
        return start.elapsed_time(stop), r

    def run(self, steps, warmup, tolerance, relative):
        for _ in range(warmup):
            self.step(tolerance, relative)
        times, results = [], []
        for _ in range(steps):
            ms, r = self.step(tolerance, relative)
            times.append(ms)
            results.append(r)
        return times, results

    def destroy(self):
        self.work.destroy()
        self.pristine.destroy()


def solved(r, tolerance, relative):
    """The solver met its stop rule (FP32 velocities may still be precision-limited)."""
    if relative:
        return r.solve_status == "converged" and r.residual_l2 <= tolerance * r.rhs_l2 * 1.0001
    return r.solve_status in ("converged", "no_work") and r.accepted()


def leg_summary(scene, times, results, tolerance, relative):
    ms = statistics.mean(times)
    iters = statistics.mean(r.iterations for r in results)
    model_bytes = scene.cells * (70 + 306 * iters)
    return {"value": scene.cells / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "iterations": iters,
            "solved": all(solved(r, tolerance, relative) for r in results),
            "converged": all(r.converged for r in results),
            "precision_limited": any(r.precision_limited for r in results),
            "max_divergence": max(r.max_divergence for r in results),
            "relative_residual": max(r.relative_residual for r in results),
            "restarts": max(r.restarts for r in results),
            "refreshes": max(r.refreshes for r in results),
            "projection_model_gbs": model_bytes / (ms / 1e3) / 1e9}


def run_cuda(args, world, rank, local_rank):
    import torch

    from fluidsim_b200 import kernel_launches
    from fluidsim_b200 import _native

    torch.cuda.set_device(local_rank)
    _native.set_launch_mode(args.launch)
    size = args.size
    scene = scene_for(size, rank)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    timer = ProjectionTimer(scene, "fp32", torch, flush, args.tail_cells)
    tail_cells, vcycle_ms, work = timer.tail_cells, timer.vcycle_ms, timer.work

    for _ in range(args.warmup):
        timer.step(args.tolerance, False)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    results, times = [], []
    launches_before = kernel_launches()
    with ClockSampler(local_rank) as clocks:
        for _ in range(args.steps):
            ms, r = timer.step(args.tolerance, False)
            times.append(ms)
            results.append(r)
    torch.cuda.synchronize()
    launches = kernel_launches() - launches_before
    total_ms = sum(times)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * scene.cells * args.steps / (total_ms / 1e3)

    # Live roofline of the fused fine-level smoothing kernels (CUDA events on the grid stream).
    peak, peak_kind = measured_peaks()
    traffic_per_cell = profiled_traffic()
    kernel_ms = {k: work.timeKernel(k, 20) for k in (0, 1)}
    dominant = max(kernel_ms, key=kernel_ms.get)
    algorithmic = ALGORITHMIC_BYTES[dominant] * scene.cells
    achieved = algorithmic / (kernel_ms[dominant] / 1e3) / 1e9
    traffic = traffic_per_cell.get(dominant)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None if traffic is None else traffic * scene.cells,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per fine cell of this kernel "
                                  "(profiles/roofline_traffic.json, a 2048x2048 capture) times the cells; "
                                  "not measured in this run",
                "kernel": KERNEL_NAMES[dominant], "kernel_ms": kernel_ms[dominant],
                "algorithmic_bytes": algorithmic, "peak_source": f"{peak_kind} hbm_gbs (copy, burst)"}
    timer.destroy()
    headline = leg_summary(scene, times, results, args.tolerance, False)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "launch": args.launch, "parallelism": f"replicas x{world}",
        "config": workload_config(size, args.tolerance),
        "iterations": headline["iterations"],
        "autotune": {"tail_cells": tail_cells, "vcycle_ms": vcycle_ms},
        "solved": headline["solved"],
        "converged": headline["converged"],
        "precision_limited": headline["precision_limited"],
        "max_divergence": headline["max_divergence"],
        "relative_residual": headline["relative_residual"],
        "restarts": headline["restarts"],
        "refreshes": headline["refreshes"],
        "roofline": roofline,
        "projection_bandwidth_model": {"iterations": headline["iterations"],
                                       "bytes": scene.cells * (70 + 306 * headline["iterations"]),
                                       "gbs": headline["projection_model_gbs"]},
        "clocks": clocks.summary(),
        "gpu_launches": launches,
    }

    if rank == 0 and not args.no_rules:
        line["relative_rule"] = rule_measure(args, scene, torch, flush, "fp32", True, tail_cells)
        line["reference_rule_fp64"] = rule_measure(args, scene, torch, flush, "fp64", False, 0)
    if rank == 0 and not args.no_mixed:
        line["mixed"] = mixed_measure(args, scene, torch, flush)
    if rank == 0 and not args.no_e2e:
        line["e2e"] = e2e_measure(args, scene, torch)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        reference = {}
        seconds, it, kind = cpu_projection(scene, args.tolerance, min(8, host_threads()), reference)
        line["cpu_baseline"] = {"value": scene.cells / seconds, "unit": UNIT, "cores": min(8, host_threads()),
                                "kind": kind, "iterations": it,
                                "sample": f"1 projection of the {size}x{size} workload"}
        if reference:
            line["error_vs_reference"] = error_vs_reference(args, scene, reference)
    if not args.no_batched:
        # Every rank projects its share of the batch (placement.py); rank 0 reports.
        batched = batched_measure(args, torch, world, rank)
        mixed = batched_measure(args, torch, world, rank, precision="mixed")
        if rank == 0:
            batched["mixed"] = {k: mixed[k] for k in ("value", "ms_per_batch", "speedup_vs_plain", "all_converged",
                                                      "max_iterations")}
            batched["mixed"]["speedup_vs_fp32"] = batched["ms_per_batch"] / mixed["ms_per_batch"]
            line["batched"] = batched
    if rank == 0 and not args.no_serve:
        line["serve"] = serve_measure(args)
    if rank == 0 and not args.no_steps:
        line["step_leg"] = steps_measure(args, torch)
        # The same 100 steps with the air held at p = 0 (the free-surface boundary the workload states).
        line["step_leg_dirichlet"] = steps_measure(args, torch, air_model="dirichlet")
    if rank == 0 and not args.no_viscous:
        from fluidsim_b200 import FluidCudaError

        try:
            line["viscous"] = viscous_measure(args, torch, flush)
        except FluidCudaError as e:  # a solver that did not converge is reported, not hidden
            line["viscous"] = {"error": str(e)}
    return line


def rule_measure(args, scene, torch, flush, precision, relative, tail_cells, steps=5, warmup=2):
    """The headline scene under another stop rule or precision: FP32 to the relative residual
    ||r|| <= tol ||b|| (the target form of the projection), and FP64 under the reference's own
    rule (the reference engine's arithmetic on the device)."""
    timer = ProjectionTimer(scene, precision, torch, flush, tail_cells, tune=tail_cells == 0)
    times, results = timer.run(steps, warmup, args.tolerance, relative)
    timer.destroy()
    out = leg_summary(scene, times, results, args.tolerance, relative)
    out["precision"] = precision
    out["stop_rule"] = "relative: ||r||_2 <= tolerance * ||b||_2" if relative else RULE
    return out


def error_vs_reference(args, scene, reference):
    """The headline step's outputs (FP32 under the reference's rule) against the reference
    engine's own FP64 outputs of the same step and rule: velocities as max |difference| over
    their scale, pressure as max |difference| over max |p| (both are mean-free)."""
    from fluidsim_b200 import FluidGrid, scenes

    g = FluidGrid(scene.width, scene.height, scene.cell_size, "fp32")
    scenes.upload_scene(g, scene)
    g.applyGravity(scene.dt)
    r = g.project(scene.dt, 400, args.tolerance)
    out = g.download()
    g.destroy()
    u, v, p = reference["u"], reference["v"], reference["p"]
    scale = max(np.abs(u).max(), np.abs(v).max())
    return {"reference": "FluidGridCPU::project, FP64, the same scene and stop rule", "device_iterations": r.iterations,
            "velocity": float(max(np.abs(out.u - u).max(), np.abs(out.v - v).max()) / scale),
            "pressure": float(np.abs(out.pressure - p).max() / np.abs(p).max())}


def mixed_measure(args, scene, torch, flush, steps=5, warmup=2):
    """The same projection in plain FP32 and in mixed precision (FP16 multigrid weights), timed
    like the main line, with the error of each against an FP64 solve of the same scene to a
    1e-12 relative residual (the device FP64 path, which matches the FP64 CPU restatement to
    1e-8 in the parity tests)."""
    from fluidsim_b200 import FluidGrid, scenes

    ref = FluidGrid(scene.width, scene.height, scene.cell_size, "fp64")
    scenes.upload_scene(ref, scene)
    ref.applyGravity(scene.dt)
    ref.project(scene.dt, 2000, 1e-12, relative_tolerance=1e-12)
    exact = ref.download()
    ref.destroy()
    scale = max(np.abs(exact.u).max(), np.abs(exact.v).max())
    out = {"fp64_reference": "device FP64 solve to 1e-12 relative"}
    for precision in ("fp32", "mixed"):
        pristine = FluidGrid(scene.width, scene.height, scene.cell_size, precision)
        scenes.upload_scene(pristine, scene)
        work = FluidGrid(scene.width, scene.height, scene.cell_size, precision)
        work.configureMaterials([scene.liquid_density], [scene.gas_density])
        work.setGravityY(scene.gravity)
        stream = torch.cuda.ExternalStream(work.stream())
        times, iters = [], []
        for i in range(warmup + steps):
            work.copyStateFrom(pristine)
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(stream)
            work.applyGravity(scene.dt)
            r = work.project(scene.dt, 200, args.tolerance, relative_tolerance=args.tolerance)
            stop.record(stream)
            stop.synchronize()
            if i >= warmup:
                times.append(start.elapsed_time(stop))
                iters.append(r.iterations)
        s = work.download()
        err = max(np.abs(s.u - exact.u).max(), np.abs(s.v - exact.v).max()) / scale
        ms = statistics.mean(times)
        out[precision] = {"value": scene.cells / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
                          "iterations": statistics.mean(iters), "velocity_error_vs_fp64": err,
                          "converged": r.solve_status == "converged"}
        work.destroy()
        pristine.destroy()
    out["speedup_vs_fp32"] = out["fp32"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["stop_rule"] = "relative: ||r||_2 <= tolerance * ||b||_2"
    return out


def e2e_measure(args, scene, torch):
    """The same step through the public API from pinned FP64 host buffers, copies included."""
    from fluidsim_b200 import FluidGrid, FluidGridState

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()

    state = FluidGridState(pinned(scene.fraction), pinned(scene.u), pinned(scene.v),
                           pinned(np.zeros_like(scene.fraction)),
                           [pinned(scene.liquid_mass[0])], [pinned(scene.gas_mass[0])])
    out = {k: pinned(np.zeros_like(a)) for k, a in (("u", scene.u), ("v", scene.v), ("p", scene.fraction))}
    g = FluidGrid(scene.width, scene.height, scene.cell_size, "fp32")
    g.configureMaterials([scene.liquid_density], [scene.gas_density])
    g.setGravityY(scene.gravity)
    stream = torch.cuda.ExternalStream(g.stream())
    import ctypes as C
    from fluidsim_b200 import _native as N

    dp = C.POINTER(C.c_double)

    def download_uvp():
        N.check(N.lib().fc_download(g.handle, None, out["u"].ctypes.data_as(dp), out["v"].ctypes.data_as(dp),
                                    out["p"].ctypes.data_as(dp), None, None))

    times = []
    for i in range(args.warmup + args.steps):
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        g.upload(state)
        g.applyGravity(scene.dt)
        g.project(scene.dt, 400, args.tolerance)
        download_uvp()
        stop.record(stream)
        stop.synchronize()
        if i >= args.warmup:
            times.append(start.elapsed_time(stop))
    n, nu, nv = scene.cells, scene.u.size, scene.v.size
    h2d = 8 * (n + nu + nv + n + 2 * n)
    d2h = 8 * (nu + nv + n)
    ms = statistics.mean(times)
    return {"value": scene.cells / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": ms, "stop_rule": RULE}


def steps_measure(args, torch, steps=100, warmup=3, size=1024, air_model="gas"):
    """Full time steps of the dam break with obstacles: a 1024x1024 scene, 16 seeded circular
    obstacles of radii 8..40 cells, gravity -9.8, dt 1/120. Each step runs RK2 semi-Lagrangian
    transport of u and v, the body force and the MG-PCG projection (FluidGrid.step, the
    reference's step order) to the 1e-6 stop rule; a step is accepted as the reference accepts
    it (converged, or precision-limited: the solver met its stop rule and only the FP32 rounding
    of the face velocities is left in the divergence). The scene evolves from step to step, timed
    with CUDA events on the grid's stream; the projection's unfused byte model gives a GB/s
    figure beside it."""
    from fluidsim_b200 import FluidGrid, scenes

    scene = scenes.dam_break(size, size, seed=11, obstacles=16, velocity=0.0)
    scene.air_model = air_model
    g = FluidGrid(size, size, scene.cell_size, "fp32")
    scenes.upload_scene(g, scene)
    stream = torch.cuda.ExternalStream(g.stream())
    times, iters, statuses, accepted = [], [], {}, True
    for i in range(warmup + steps):
        with torch.cuda.stream(stream):
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
        r = g.step(scene.dt, 200, args.tolerance)
        stop.record(stream)
        stop.synchronize()
        if i >= warmup:
            times.append(start.elapsed_time(stop))
            iters.append(r.iterations)
            statuses[r.solve_status] = statuses.get(r.solve_status, 0) + 1
            accepted = accepted and r.accepted()
    g.destroy()
    ms = statistics.mean(times)
    mean_iters = statistics.mean(iters)
    model_bytes = scene.cells * (70 + 306 * mean_iters)
    return {"workload": f"dam_break_{size}x{size}, 16 obstacles, {steps} steps after {warmup}", "air_model": air_model,
            "value": scene.cells / (ms / 1e3),
            "unit": UNIT, "ms_per_step": ms, "p50_ms": statistics.median(times), "max_ms": max(times),
            "iterations_per_step": mean_iters, "max_iterations": max(iters), "solve_status": statuses,
            "all_accepted": accepted,
            "projection_model_gbs": model_bytes / (ms / 1e3) / 1e9}


def viscous_measure(args, torch, flush, size=4096, steps=3, warmup=1):
    """Variable-viscosity flow at 4096x4096 (scenes.viscous_blob: a fractal liquid blob over 60 %
    of the domain, 1000:1 density ratio, viscosity log-uniform in [1e-3, 10] along a smooth noise
    field, U[-1, 1] FP32 velocities). One step is the implicit viscosity solve (V-cycle
    preconditioned CG to the reference's 1e-4 relative residual) and then the MG-PCG projection
    to the 1e-6 stop rule, from the same initial state every time, timed with CUDA events on the
    grid's stream after an L2 flush. Plain FP32 and mixed precision (FP16 coarse-level pressure
    weights) are each compared with an FP64 device solve of the same step: the viscosity to the
    same 1e-4 stop rule (a tighter viscosity solve moves the velocities by a few percent of their
    scale, which would hide the precision), then the pressure to a 1e-12 relative residual."""
    from fluidsim_b200 import FluidGrid, scenes

    scene = scenes.viscous_blob(size, size, seed=5)
    ref = FluidGrid(size, size, scene.cell_size, "fp64")
    scenes.upload_scene(ref, scene)
    ref_visc, _ = ref.applyViscosity(scene.dt, 1e-4, 4000)
    ref_proj = ref.project(scene.dt, 4000, 1e-12, relative_tolerance=1e-12)
    exact = ref.download()
    ref.destroy()
    scale = max(np.abs(exact.u).max(), np.abs(exact.v).max())
    out = {"workload": f"viscous_blob_{size}x{size}: viscosity then projection, {steps} steps after {warmup}",
           "fp64_reference": {"viscosity_iterations": ref_visc, "pressure_iterations": ref_proj.iterations,
                              "tolerances": "viscosity 1e-4 (the reference's rule), pressure 1e-12 relative"}}
    for precision in ("fp32", "mixed"):
        pristine = FluidGrid(size, size, scene.cell_size, precision)
        scenes.upload_scene(pristine, scene)
        work = FluidGrid(size, size, scene.cell_size, precision)
        scenes.configure_grid(work, scene)
        stream = torch.cuda.ExternalStream(work.stream())
        total, visc_ms, visc_it, proj_it = [], [], [], []
        for i in range(warmup + steps):
            work.copyStateFrom(pristine)
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                events = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                events[0].record(stream)
            it, _ = work.applyViscosity(scene.dt, 1e-4, 4000)
            events[1].record(stream)
            r = work.project(scene.dt, 400, args.tolerance, relative_tolerance=args.tolerance)
            events[2].record(stream)
            events[2].synchronize()
            if i >= warmup:
                total.append(events[0].elapsed_time(events[2]))
                visc_ms.append(events[0].elapsed_time(events[1]))
                visc_it.append(it)
                proj_it.append(r.iterations)
        s = work.download()
        err = max(np.abs(s.u - exact.u).max(), np.abs(s.v - exact.v).max()) / scale
        ms = statistics.mean(total)
        out[precision] = {"value": scene.cells / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
                          "viscosity_ms": statistics.mean(visc_ms), "viscosity_iterations": statistics.mean(visc_it),
                          "pressure_iterations": statistics.mean(proj_it), "pressure_status": r.solve_status,
                          "relative_residual": r.relative_residual, "velocity_error_vs_fp64": err}
        work.destroy()
        pristine.destroy()
    out["speedup_vs_fp32"] = out["fp32"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    return out


def batched_measure(args, torch, world=1, rank=0, count=256, precision="fp32"):
    """Uneven grids (sides log-uniform 64..1024, aspect <= 2:1, fill 0.3-0.9, 0-8 obstacles)
    projected together, against the same grids projected one at a time. With several ranks the
    grids are placed whole on the ranks (no exchange between them) and the slowest rank's time
    is reported."""
    from fluidsim_b200 import FluidGrid, ProjectionBatch, scenes
    from fluidsim_b200.placement import max_over_ranks, mine, place
    from fluidsim_b200.serving import grid_device_bytes

    all_scenes = scenes.uneven_batch(count, seed=7)
    total_cells = sum(s.cells for s in all_scenes)
    assignment = place([s.cells for s in all_scenes],
                       [2 * grid_device_bytes(s.width, s.height) for s in all_scenes], world, 150 * 10**9)
    batch_scenes = [all_scenes[i] for i in mine(assignment, rank)]
    grids, pristine = [], []
    for s in batch_scenes:
        p = FluidGrid(s.width, s.height, s.cell_size, precision)
        scenes.upload_scene(p, s)
        g = FluidGrid(s.width, s.height, s.cell_size, precision)
        g.configureMaterials([s.liquid_density], [s.gas_density])
        g.setObstacles(s.solid)
        pristine.append(p)
        grids.append(g)
    cells = sum(s.cells for s in batch_scenes)
    batch = ProjectionBatch(grids)
    dts = [s.dt for s in batch_scenes]
    for g, p in zip(grids, pristine):
        g.copyStateFrom(p)
    tail_cells, _ = batch.autotune(5)

    def restore():
        for g, p in zip(grids, pristine):
            g.copyStateFrom(p)

    stream = torch.cuda.ExternalStream(batch.stream())
    times = []
    for i in range(2 + 3):
        restore()
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        res = batch.project(dts, 300, args.tolerance, relative_tolerance=args.tolerance)
        stop.record(stream)
        stop.synchronize()
        if i >= 2:
            times.append(start.elapsed_time(stop))
    batched_ms = statistics.mean(times)
    ok = all(r.solve_status in ("converged", "no_work") for r in res)
    # One grid at a time through the same engine (the plain path).
    restore()
    torch.cuda.synchronize()
    plain_ms = 0.0
    for g in grids:
        gs = torch.cuda.ExternalStream(g.stream())
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(gs)
        g.project(dts[grids.index(g)], 300, args.tolerance, relative_tolerance=args.tolerance)
        stop.record(gs)
        stop.synchronize()
        plain_ms += start.elapsed_time(stop)
    batch.destroy()
    dev = torch.device("cuda", torch.cuda.current_device())
    batched_ms = max_over_ranks(batched_ms, dev)
    plain_ms = max_over_ranks(plain_ms, dev)
    ok = max_over_ranks(0.0 if ok else 1.0, dev) == 0.0
    return {"value": total_cells / (batched_ms / 1e3), "unit": UNIT, "precision": precision, "grids": count,
            "cells": total_cells,
            "ranks": world, "ms_per_batch": batched_ms,
            "plain_one_at_a_time_cells_per_s": total_cells / (plain_ms / 1e3),
            "speedup_vs_plain": plain_ms / batched_ms, "all_converged": ok, "tail_cells": tail_cells,
            "max_iterations": max(r.iterations for r in res)}


SERVE_CLASSES = (128 * 128, 256 * 256, 512 * 512, 1024 * 1024)  # the server's default size classes (cells)


def serve_measure(args, rate=200.0, budget=150 * 10**9, precision="mixed"):
    """Serving: Poisson arrivals (mean `rate` per second) of dam breaks with surface tension
    (sigma 0.07, liquid 1000, air 1), square sides log-uniform 64..2048, each run for
    serve_steps steps of dt 1/120 to the max-norm rule at the bench tolerance, in mixed
    precision, admitted by a device-memory budget and batched as they arrive in five size
    classes (up to 128^2, 256^2, 512^2, 1024^2 cells, larger), each stepped by its own worker. The same
    simulations are then run one at a time through fc_step (the plain path, same precision).
    Step latencies are reported per size class for both. A bounded sample: serve_requests
    requests."""
    import time

    from fluidsim_b200 import FluidGrid, scenes
    from fluidsim_b200.serving import Server, poisson_arrivals, serve

    reqs = scenes.serving_requests(args.serve_requests, seed=5)
    arrivals = poisson_arrivals(rate, len(reqs), seed=6)
    steps = args.serve_steps
    cell_steps = steps * sum(s.cells for s in reqs)
    # The served form runs three times (a fresh server each); the run of median wall time is
    # reported, and every run's wall time is listed.
    runs = []
    for _ in range(3):
        server = Server(budget, max_active=256)
        out = serve(server, reqs, arrivals, steps, 200, args.tolerance, precision=precision)
        stats, per_class = server.stats(), server.class_stats()
        failures = [{"side": s.width, "state": st.state, "error": server.error(sim)}
                    for s, sim, st in zip(reqs, out["ids"], out["statuses"]) if st.state != "done"]
        if failures:
            print(f"bench.py: served simulations failed: {failures}", file=sys.stderr)
        for sim in out["ids"]:
            server.release(sim)
        server.close()
        runs.append((out["wall_s"], out, stats, per_class, failures))
    walls = [r[0] for r in runs]
    _, out, stats, per_class, failures = sorted(runs, key=lambda r: r[0])[1]
    served_ok = not any(r[4] for r in runs)

    def size_class(cells):
        return sum(cells > b for b in SERVE_CLASSES)

    plain_lat = [[] for _ in range(len(SERVE_CLASSES) + 1)]
    plain_class_s = [0.0] * (len(SERVE_CLASSES) + 1)
    t0 = time.perf_counter()
    for s in reqs:
        k = size_class(s.cells)
        a0 = time.perf_counter()
        g = FluidGrid(s.width, s.height, s.cell_size, precision)
        scenes.upload_scene(g, s)
        for _ in range(steps):
            a = time.perf_counter()
            g.step(s.dt, 200, args.tolerance)
            plain_lat[k].append((time.perf_counter() - a) * 1e3)
        g.destroy()
        plain_class_s[k] += time.perf_counter() - a0
    plain_s = time.perf_counter() - t0

    def pct(a, q):
        a = np.sort(np.asarray(a))
        return float(a[max(0, int(np.ceil(q * len(a))) - 1)]) if len(a) else None

    classes = []
    for k, c in enumerate(per_class):
        members = [s for s in reqs if size_class(s.cells) == k]
        classes.append({"max_cells": c["max_cells"] if k < len(SERVE_CLASSES) else None,
                        "sizes": sorted(s.width for s in members),
                        "served": {"step_p50_ms": c["step_p50_ms"], "step_p99_ms": c["step_p99_ms"],
                                   "step_max_ms": c["step_max_ms"], "ticks": c["ticks"], "busy_s": c["busy_ms"] / 1e3},
                        "plain": {"step_p50_ms": pct(plain_lat[k], 0.5), "step_p99_ms": pct(plain_lat[k], 0.99),
                                  "wall_s": plain_class_s[k]}})
    every = [x for lat in plain_lat for x in lat]
    served = cell_steps / out["wall_s"]
    plain = cell_steps / plain_s
    return {"value": served, "unit": UNIT, "precision": precision, "requests": len(reqs), "steps_per_request": steps,
            "arrival_rate_per_s": rate, "sizes": sorted(s.width for s in reqs),
            "sample": f"{len(reqs)} requests (bounded sample of the Poisson stream), sides log-uniform 64..2048, "
                      f"dx 1/128, sigma 0.07, dt 1/120",
            "wall_s": out["wall_s"], "wall_s_runs": walls, "step_p50_ms": stats["step_p50_ms"], "step_p99_ms": stats["step_p99_ms"],
            "step_max_ms": stats["step_max_ms"], "peak_active": stats["peak_active"],
            "peak_device_bytes": stats["peak_bytes"], "budget_bytes": budget, "batch_plans_built": stats["batch_rebuilds"],
            "all_done": served_ok, "failures": failures, "size_classes": classes,
            "plain": {"value": plain, "unit": UNIT, "wall_s": plain_s, "step_p50_ms": pct(every, 0.5),
                      "step_p99_ms": pct(every, 0.99)},
            "speedup_vs_plain": served / plain}


def spawn_ranks(args):
    """Runs this script under torch.distributed.run with one rank per GPU (the caller asked
    for N > 1 GPUs without starting the ranks); returns its exit code."""
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(spawn_ranks(args))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE is {world}", file=sys.stderr)
        sys.exit(2)
    if args.impl == "reference":
        line = run_reference(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    line = run_cuda(args, world, rank, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
