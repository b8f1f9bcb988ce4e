"""Benchmark of the liquid substep on B200.

Workload: the sparse 256^3 splash (pool y <= 0.2 over the floor + two
counter-moving spheres), 8 particles per fluid cell (~29.6M particles), FP32
transfers, mixed-precision projection (BF16 V-cycle storage, FP32 flexible CG,
FP64 refinement to a 1e-6 relative residual). One step = topology + sort + P2G
(+normalize, gravity, walls) + projection + G2P (+advection). Data: seeded
synthetic scene generated on the host (no dataset involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0). With N > 1 (torchrun) every rank runs an
independent replica: the path has no data exchange between GPUs.
"""

from __future__ import annotations

import argparse
import atexit
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "steps/s at 256^3 APIC (sparse splash, ~29.6M particles, projection to 1e-6 relative residual)"
UNIT = "steps/s"
SCENES = {
    "splash": "pool y<=0.2 + two r=0.15 spheres at +-2 m/s",
    "column_drop": "column [0.1,0.3]x[0.1,0.8]x[0.1,0.3] falling into a pool y<=0.15",
}


def workload(scene: str, grid: int, precision: int):
    return {"workload": f"{scene}_{grid}", "grid": grid, "scene": SCENES[scene], "particles_per_cell": 8,
            "dt": 1.0 / 240.0,
            "precision": "fp32 transfers, " + ("bf16" if precision else "fp32") + " V-cycle storage (the other "
                         "measured beside), fp32 FCG, fp64 refinement",
            "rel_tol": 1e-6, "l2": "inputs (particles, GBs) larger than the 126 MB L2; no flush"}
FALLBACK_HBM_GBS = 6650.0


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's time: every rank contributes its own device-timed
    milliseconds and all receive the maximum (identity on one rank). Replicas
    exchange nothing else."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, steps: int, max_ms: float) -> float:
    """Weak-scaling throughput: every replica advances `steps` steps of its own
    scene, so the job completes world * steps steps in the slowest rank's time."""
    return world * steps / (max_ms / 1e3)


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons every 50 ms. The
    sampler starts before the warm-up (nvidia-smi takes a moment to come up) and
    only the samples stamped inside the timed window (mark_start / mark_stop)
    are summarised."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def mark_start(self):
        self.t0 = datetime.datetime.now()

    def mark_stop(self):
        self.t1 = datetime.datetime.now()

    def __exit__(self, *exc):
        if self.proc is not None:  # idempotent: also called on error paths
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.proc = None

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = [r.split(",") for r in Path(self.path).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                ts = datetime.datetime.strptime(r[0].strip(), "%Y/%m/%d %H:%M:%S.%f")
                if self.t0 is not None and self.t1 is not None and not (self.t0 <= ts <= self.t1):
                    continue
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, name in enumerate(names):
                    if r[4 + k].strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _traffic_per_launch(particles: int, cells: int):
    """DRAM bytes of one P2G launch pair from the committed ncu summary, scaled
    by the units processed (profiles/p2g_splash.md records bytes per particle)."""
    prof = ROOT / "profiles" / "p2g_splash.md"
    if not prof.exists():
        return None
    for line in prof.read_text().splitlines():
        if line.startswith("traffic_bytes_per_particle:"):
            return float(line.split(":")[1]) * particles
    return None


# Algorithmic bytes per allocated cell (active blocks x 512) of one flexible-CG
# iteration, each array element counted once per kernel, V-cycle x and
# coefficients in BF16:
#   k_dots 10 (z, r, r_prev) + k_direction_tiled 15 (z, d_old, mask -> d, q)
#   + k_update 24 (d, q, r, e -> e, r_next)                                   = 49
#   level 0, per sweep the colour's mask, b and diag, the other colour's x and
#   the colour's x written: the from-zero sweep 5.5, a sweep 6.5, the
#   prolongation sweep 6.75; the restriction 11.9 (mask, diag, b, x; coarse b
#   and seed). With `pre` pre- and `post` post-smoothing sweeps:
#   5.5 + 6.5 + 13 (pre - 1) + 6.75 + 6.5 (2 post - 1) + 11.9
#   (63.2 for two and two, 50.2 for one and two)
#   levels >= 1: ~106 B per coarse cell per V-cycle at two and two, 1/8 per
#   level (15.5), scaled with level 0's sweeps
# FP32 storage reads x and the coefficients at 4 B: the V-cycle part x 109/78.65
# (158 B in all for two and two, against 128 in BF16).
def _pressure_bytes_per_cell_iter(precision: int, pre: int, post: int) -> float:
    level0 = 5.5 + 6.5 + 13.0 * (pre - 1) + 6.75 + 6.5 * (2 * post - 1) + 11.9
    vcycle = level0 + 15.5 * level0 / 63.15
    if precision == 0:
        vcycle *= 109.0 / 78.65
    return round(49.0 + vcycle, 1)


def _pressure_roofline(cells: int, iterations: float, pressure_ms: float, peak: float, precision: int,
                       pre: int, post: int):
    """Iteration bytes over the whole projection's time (setup, FP64 residuals,
    correction and export included in the time but not in the bytes): a lower
    bound on the solver's achieved bandwidth."""
    per = _pressure_bytes_per_cell_iter(precision, pre, post)
    moved = per * cells * iterations
    achieved = moved / (pressure_ms / 1e3) / 1e9
    return {"bytes_per_cell_per_iteration": per, "cells": cells, "iterations": iterations,
            "algorithmic_bytes": int(moved), "achieved": round(achieved, 1), "frac": round(achieved / peak, 4)}


def run_ours(args, world, rank, local):
    import torch

    import fluidity_b200 as fb
    from fluidity_b200 import scenes

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    soa, mass = scenes.SCENES[args.scene](args.grid)
    npart = soa.shape[1]
    ctx = fb.LiquidContext(args.grid, capacity=npart)
    tp = fb.transfer_params(scenes.DT, mass)
    opt = fb.default_pressure_options(precision=args.precision, rel_tol=1e-6, warm_start=1, inner_rtol=1e-3)
    ctx.upload(soa)
    clocks = ClockSampler(local).__enter__()
    atexit.register(clocks.__exit__, None, None, None)  # never leave nvidia-smi running
    for _ in range(args.warmup):
        code, _ = ctx.step(tp, opt)
    torch.cuda.synchronize()
    nb_first = len(ctx.active_blocks())
    if world > 1:
        torch.distributed.barrier()
    launches0 = fb.kernel_launches()
    phases = np.zeros(4)
    iters = []
    residuals = []
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clocks.mark_start()
    start.record()
    for _ in range(args.steps):
        code, diag = ctx.step(tp, opt)
        phases += ctx.step_timings()
        iters.append(diag.iterations)
        residuals.append(diag.relative_residual)
        if code != fb.OK:
            raise RuntimeError(f"pressure did not converge: {diag.as_dict()}")
    stop.record()
    torch.cuda.synchronize()
    clocks.mark_stop()
    clocks.__exit__(None, None, None)
    launches1 = fb.kernel_launches()
    ms = start.elapsed_time(stop)
    nb_last = len(ctx.active_blocks())
    # the other V-cycle storage precision on the same steps: restart from the initial state
    alt_prec = 1 - args.precision
    alt_opt = fb.default_pressure_options(precision=alt_prec, rel_tol=1e-6, warm_start=1, inner_rtol=1e-3)
    alt_phases, alt_iters = np.zeros(4), []
    ctx.upload(soa)
    for _ in range(args.warmup):
        ctx.step(tp, alt_opt)
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a0.record()
    for _ in range(args.steps):
        code, diag = ctx.step(tp, alt_opt)
        alt_phases += ctx.step_timings()
        alt_iters.append(diag.iterations)
        if code != fb.OK:
            raise RuntimeError(f"pressure did not converge: {diag.as_dict()}")
    a1.record()
    torch.cuda.synchronize()
    alt_ms = a0.elapsed_time(a1) / args.steps
    ms = max_over_ranks(ms, world)
    ms_per_step = ms / args.steps
    value = whole_job_rate(world, args.steps, ms)
    # allocated cells over the timed steps (the splash spreads): the mean of the first and last counts
    ncell = (nb_first + nb_last) // 2 * 512
    # End to end through the C-ABI from pinned host memory, every step: the H2D
    # copy of the step's input (staged on the context's own stream one step
    # ahead, so it runs beside the step before it), the step, and the D2H of its
    # result through the snapshot queue (device check + copy on the queue's
    # stream, beside the next step), finished and read on the host.
    pin_in = torch.from_numpy(soa).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    host_in, host_out = pin_in.numpy(), pin_out.numpy()
    queue = fb.SnapshotQueue(ctx)
    e2e_steps = max(2, min(args.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    probe = 0.0

    def take(ticket):
        nonlocal probe
        if queue.wait(ticket) != fb.SNAPSHOT_READY:
            raise RuntimeError("snapshot did not complete")
        out, _ = queue.finish(ticket)
        probe += float(out[0, 0]) + float(out[14, -1])  # the host reads the result
        queue.release(ticket)

    # the first staging allocates the context's two extra particle buffers: done
    # once before the timed region (the upload drops the staged input)
    ctx.stage(host_in)
    ctx.upload(host_in)
    torch.cuda.synchronize()
    e0.record()
    prev = None
    ctx.stage(host_in)
    for k in range(e2e_steps):
        if k + 1 < e2e_steps:
            ctx.stage(host_in)  # the next step's input
        code, diag = ctx.step(tp, opt)
        if code != fb.OK:
            raise RuntimeError(f"pressure did not converge: {diag.as_dict()}")
        ticket = queue.begin(k + 1, k + 1, (k + 1) * scenes.DT)
        if prev is not None:
            take(prev)
        prev = ticket
    take(prev)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, world)
    queue.close()
    # the same through the synchronous host step (fl_step_host: H2D, step, D2H in turn)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s0.record()
    for _ in range(e2e_steps):
        ctx.step_host(host_in, host_out, tp, opt)
    s1.record()
    torch.cuda.synchronize()
    e2e_sync_ms = max_over_ranks(s0.elapsed_time(s1) / e2e_steps, world)
    peak, peak_kind = _peaks()
    p2g_ms = phases[1] / args.steps
    p2g_bytes = 60.0 * npart + 24.0 * ncell
    achieved = p2g_bytes / (p2g_ms / 1e3) / 1e9
    g2p_ms = phases[3] / args.steps
    g2p_bytes = 72.0 * npart + 12.0 * ncell
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": f"synthetic (seeded {args.scene} scene)",
        "config": dict(workload(args.scene, args.grid, args.precision), particles=npart,
                       active_blocks=[nb_first, nb_last], allocated_cells=ncell, timed_steps=[args.warmup + 1,
                                                                                      args.warmup + args.steps],
                       parallelism=f"replicas{world}"),
        "e2e": {"value": round(world * 1e3 / e2e_ms, 4), "unit": UNIT, "h2d_bytes_per_step": int(60 * npart),
                "d2h_bytes_per_step": int(60 * npart + 64), "steps": e2e_steps,
                "path": "fl_stage_particles (one step ahead) -> fl_step -> fl_snapshot_begin/wait/finish "
                        "(H2D, step and D2H of consecutive steps overlap)"},
        "e2e_sync": {"value": round(world * 1e3 / e2e_sync_ms, 4), "unit": UNIT,
                     "h2d_bytes_per_step": int(60 * npart), "d2h_bytes_per_step": int(60 * npart),
                     "path": "fl_step_host (H2D, step, D2H in turn)"},
        "roofline": {"kernel": "p2g (k_p2g_tile + k_p2g_merge)", "bound": "hbm", "achieved": round(achieved, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "algorithmic_bytes": int(p2g_bytes), "traffic": _traffic_per_launch(npart, ncell)},
        "phases_ms": {"topology_sort": round(phases[0] / args.steps, 4), "p2g": round(p2g_ms, 4),
                      "pressure": round(phases[2] / args.steps, 4), "g2p": round(g2p_ms, 4)},
        "g2p_roofline": {"achieved": round(g2p_bytes / (g2p_ms / 1e3) / 1e9, 1), "frac": round(
            g2p_bytes / (g2p_ms / 1e3) / 1e9 / peak, 4)},
        "transfers_roofline": {"kernels": "P2G + G2P", "algorithmic_bytes": int(p2g_bytes + g2p_bytes),
                               "achieved": round((p2g_bytes + g2p_bytes) / ((p2g_ms + g2p_ms) / 1e3) / 1e9, 1),
                               "frac": round((p2g_bytes + g2p_bytes) / ((p2g_ms + g2p_ms) / 1e3) / 1e9 / peak, 4)},
        "pressure_roofline": _pressure_roofline(ncell, float(np.mean(iters)), phases[2] / args.steps, peak,
                                                args.precision, opt.pre_sweeps, opt.post_sweeps),
        "particles_per_s": round(value * npart, 1),
        "pressure": {"mean_iterations": float(np.mean(iters)), "max_relative_residual": float(max(residuals)),
                     "vcycle_storage": "bf16" if args.precision == 1 else "fp32", "inner_rtol": 1e-3},
        "vcycle_" + ("bf16" if alt_prec == 1 else "fp32"): {
            "steps_per_s": round(1e3 / alt_ms, 4), "ms_per_step": round(alt_ms, 4),
            "pressure_ms": round(alt_phases[2] / args.steps, 4), "mean_iterations": float(np.mean(alt_iters))},
        "gpu_launches": int(launches1[0] - launches0[0]),
        "library_launches": int(launches1[1] - launches0[1]),
        "clocks": clocks.summary(),
    }
    learned_params = None
    if not args.no_learned:
        line["pressure_solve_ms"], learned_params = pressure_comparison(ctx, tp, args.grid)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(soa, mass, args.grid, npart, ncell, budget_s=args.cpu_budget)
        # One more step of the same run, outside every timed region, replayed
        # field by field by the FP64 oracle on the host (the checker).
        line["parity_vs_fp64"] = parity_vs_fp64(ctx, tp, opt, args.grid, args.warmup + args.steps + 1)
    ctx.close()
    if world == 1 and not args.no_column_drop:
        line["column_drop_512"] = column_drop_512(peak, learned_params)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return line


def column_drop_512(peak, learned_params, steps=5, warmup=3):
    """The 512^3 column drop (column [0.1,0.3]x[0.1,0.8]x[0.1,0.3] over a pool
    y <= 0.15, 8 particles per fluid cell) on the same GPU after the headline:
    steps/s and particles/s over `steps` CUDA-event-timed steps after `warmup`,
    the phase times and rooflines as for the headline, and the pressure solve
    of the last step's projection from p = 0 to a 1e-6 FP64 relative residual
    with plain FP32 MGPCG, BF16-storage MGPCG and the learned preconditioner."""
    import torch

    import fluidity_b200 as fb
    from fluidity_b200 import scenes

    t0 = time.time()
    soa, mass = scenes.column_drop(512)
    npart = soa.shape[1]
    gen_s = time.time() - t0
    ctx = fb.LiquidContext(512, capacity=npart)
    tp = fb.transfer_params(scenes.DT, mass)
    opt = fb.default_pressure_options(precision=1, rel_tol=1e-6, warm_start=1, inner_rtol=1e-3)
    ctx.upload(soa)
    fluid_cells = npart // 8
    del soa
    for _ in range(warmup):
        code, _ = ctx.step(tp, opt)
    nb0 = len(ctx.active_blocks())
    phases, iters = np.zeros(4), []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        code, d = ctx.step(tp, opt)
        if code != fb.OK:
            raise RuntimeError(f"column drop: pressure did not converge: {d.as_dict()}")
        phases += ctx.step_timings()
        iters.append(d.iterations)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    nb1 = len(ctx.active_blocks())
    ncell = (nb0 + nb1) // 2 * 512
    p2g_ms, g2p_ms, pr_ms = phases[1] / steps, phases[3] / steps, phases[2] / steps
    tb = 132.0 * npart + 36.0 * ncell
    out = {"workload": "column_drop_512", "grid": 512, "particles": npart, "fluid_cells_initial": fluid_cells,
           "active_blocks": [nb0, nb1], "allocated_cells": ncell, "steps": steps, "warmup": warmup,
           "steps_per_s": round(1e3 / ms, 3), "ms_per_step": round(ms, 3),
           "particles_per_s": round(npart * 1e3 / ms, 1),
           "phases_ms": {"topology_sort": round(phases[0] / steps, 3), "p2g": round(p2g_ms, 3),
                         "pressure": round(pr_ms, 3), "g2p": round(g2p_ms, 3)},
           "transfers_roofline": {"algorithmic_bytes": int(tb),
                                  "achieved": round(tb / ((p2g_ms + g2p_ms) / 1e3) / 1e9, 1),
                                  "frac": round(tb / ((p2g_ms + g2p_ms) / 1e3) / 1e9 / peak, 4)},
           "pressure_roofline": _pressure_roofline(ncell, float(np.mean(iters)), pr_ms, peak, 1, opt.pre_sweeps,
                                                   opt.post_sweeps),
           "mean_iterations": float(np.mean(iters)), "scene_seconds": round(gen_s, 1),
           "data": "synthetic (seeded column_drop scene, generated on the host z-slab by z-slab)"}
    variants = {"mgpcg_fp32": dict(precision=0), "mgpcg_bf16": dict(precision=1)}
    if learned_params is not None:
        ctx.set_learned_preconditioner(learned_params)
        variants["learned_bf16"] = dict(precision=1, preconditioner=1)
        variants["learned_composite_bf16"] = dict(precision=1, preconditioner=2)
    solve = {"unit": "ms", "relative_residual": 1e-6, "start": "p = 0"}
    for name, kw in variants.items():
        best = None
        for _ in range(2):
            code, d = ctx.project(tp, fb.default_pressure_options(rel_tol=1e-6, warm_start=0, **kw))
            if code != fb.OK:
                raise RuntimeError(f"column drop {name}: pressure did not converge: {d.as_dict()}")
            if best is None or d.solve_ms < best.solve_ms:
                best = d
        solve[name] = {"ms": round(best.solve_ms, 3), "iterations": best.iterations,
                       "learned_iterations": best.learned_iterations, "fell_back": best.fell_back,
                       "relative_residual": best.relative_residual}
    if "learned_bf16" in solve:
        solve["learned_vs_fp32_mgpcg_speedup"] = round(solve["mgpcg_fp32"]["ms"] / solve["learned_bf16"]["ms"], 3)
        solve["composite_vs_fp32_mgpcg_speedup"] = round(
            solve["mgpcg_fp32"]["ms"] / solve["learned_composite_bf16"]["ms"], 3)
    out["pressure_solve_ms"] = solve
    ctx.close()
    return out


def parity_vs_fp64(ctx, tp, opt, grid, step_number):
    """Errors of one device step of the workload against its FP64 replay
    (oracle.replay.step_parity): the state before the step is downloaded, the
    device runs the step, and the oracle repeats it on the host with the
    device's pressure; u_pred/u_new/v/C norm-wise relative, x in cells, the
    pressure as its FP64 relative residual on the device's own system."""
    from fluidity_b200 import scenes
    from oracle.replay import step_parity

    import fluidity_b200 as fb

    t0 = time.time()
    state = ctx.download()
    ctx.upload(state)
    code, diag = ctx.step(tp, opt)
    if code != fb.OK:
        return {"error": f"step failed: {diag.as_dict()}"}
    blocks = ctx.active_blocks()
    nb = len(blocks)
    f = ctx.fields()
    nn = (grid, grid, grid)
    fields = {
        "u_pred": [fb.sparse_faces_to_dense(blocks, fb.copy_to_host(f["u_pred"][a], nb * 512, np.float32), nn, a,
                                            fill=np.nan) for a in range(3)],
        "u_new": [fb.sparse_faces_to_dense(blocks, fb.copy_to_host(f["u_new"][a], nb * 512, np.float32), nn, a,
                                           fill=np.nan) for a in range(3)],
        "pressure": fb.sparse_cells_to_dense(blocks, fb.copy_to_host(f["pressure"], nb * 512, np.float64), nn,
                                             fill=np.nan),
        "cell_type": fb.sparse_cells_to_dense(blocks, fb.copy_to_host(f["cell_type"], nb * 512, np.uint8), nn,
                                              fill=255),
    }
    out = ctx.download()
    errs = step_parity(grid, state, out, fields, scenes.DT)
    errs = {k: (round(v, 12) if isinstance(v, float) else v) for k, v in errs.items()}
    errs.update({"step": step_number, "vcycle_storage": "bf16" if opt.precision == 1 else "fp32",
                 "device_relative_residual": diag.relative_residual, "tolerance": 1e-5,
                 "seconds": round(time.time() - t0, 1),
                 "how": "FP64 replay (oracle/cpu fo_step_replay) of one device step from the device's state with "
                        "the device's pressure: grid fields on every face, particle fields on every 61st particle"})
    return errs


def pressure_comparison(ctx, tp, grid, repeats=2):
    """Pressure-solve time to a 1e-6 relative FP64 residual on the last step's
    projection, each variant from p = 0 (no warm start): plain FP32 MGPCG, the
    BF16-storage V-cycle, and the learned block preconditioner (trained here on
    the residual windows of 128^3 dam-break solves to invert the pressure
    operator on its block): in place of the V-cycle with the V-cycle as
    fallback (learned_bf16), and as a correction added after each V-cycle
    (learned_composite_bf16). Times are the solver's own CUDA events (setup +
    iterations + velocity correction); the minimum over `repeats` runs."""
    import time

    import fluidity_b200 as fb
    from fluidity_b200 import learned

    t0 = time.time()
    x, t, m = learned.collect_pairs(128, 10000)
    P, losses = learned.train(x, t, m, steps=2000, batch=64, lr=1e-3)
    train_s = time.time() - t0
    ctx.set_learned_preconditioner(P)
    variants = {
        "mgpcg_fp32": dict(precision=0),
        "mgpcg_bf16": dict(precision=1),
        "learned_bf16": dict(precision=1, preconditioner=1),
        "learned_composite_bf16": dict(precision=1, preconditioner=2),
    }
    out = {"unit": "ms", "relative_residual": 1e-6, "start": "p = 0", "grid": grid}
    for name, kw in variants.items():
        best = None
        for _ in range(repeats):
            code, d = ctx.project(tp, fb.default_pressure_options(rel_tol=1e-6, warm_start=0, **kw))
            if code != fb.OK:
                raise RuntimeError(f"{name}: pressure did not converge: {d.as_dict()}")
            if best is None or d.solve_ms < best.solve_ms:
                best = d
        out[name] = {"ms": round(best.solve_ms, 3), "iterations": best.iterations,
                     "learned_iterations": best.learned_iterations, "fell_back": best.fell_back,
                     "relative_residual": best.relative_residual}
    out["learned_vs_fp32_mgpcg_speedup"] = round(out["mgpcg_fp32"]["ms"] / out["learned_bf16"]["ms"], 3)
    out["composite_vs_fp32_mgpcg_speedup"] = round(out["mgpcg_fp32"]["ms"] / out["learned_composite_bf16"]["ms"], 3)
    out["training"] = {"pairs": int(x.shape[0]), "adam_steps": 2000, "batch": 64, "lr": 1e-3,
                       "loss": "block residual |r_b - A_b y|^2 / max(|r_b|^2, 1) (zero correction <= 1)",
                       "seconds": round(train_s, 1), "loss_first": float(losses[:20].mean()),
                       "loss_last": float(losses[-20:].mean())}
    return out, P


def _sample_cube(soa, grid, sample):
    """Particles inside an axis-aligned cube in the pool, sized to hold about
    `sample` particles (8 per cell), centred away from the walls."""
    half = 0.5 * (sample / (8.0 * grid ** 3)) ** (1.0 / 3.0)
    centre = np.array([0.5, min(0.1, 0.2 - half), 0.5])
    x = soa[0:3].T
    inside = np.all(np.abs(x - centre) <= half, axis=1)
    return np.nonzero(inside)[0]


def _reference_sample_times(soa, mass, grid, sample, threads):
    """Times the reference's own CPU operators (compiled from source) on a
    compact particle sample split over `threads` host threads, plus one
    ProjectMacPressure3D at its 4096-cell capacity."""
    import oracle
    from concurrent.futures import ThreadPoolExecutor

    if oracle.ref() is None:
        return None
    h = 1.0 / grid
    idx = _sample_cube(soa, grid, sample)
    x = soa[0:3, idx].T.astype(np.float64)
    v = soa[3:6, idx].T.astype(np.float64)
    c = soa[6:15, idx].T.astype(np.float64)
    order = np.argsort(x[:, 0], kind="stable")
    x, v, c = x[order], v[order], c[order]
    chunks = [ch for ch in np.array_split(np.arange(len(idx)), threads) if len(ch)]
    jobs = []
    for ch in chunks:
        xs = x[ch]
        lo = np.floor(xs.min(0) / h / 4).astype(int) - 1
        hi = np.floor(xs.max(0) / h / 4).astype(int) + 1
        blocks = np.array([[i, j, k] for k in range(lo[2], hi[2] + 1) for j in range(lo[1], hi[1] + 1)
                           for i in range(lo[0], hi[0] + 1)], np.int32)
        jobs.append((blocks, oracle.particles_aos(xs, v[ch], c[ch], mass)))

    def work(job):
        blocks, parts = job
        oracle.ref_deposit([0, 0, 0], h, blocks, parts)
        u = np.zeros(192 * len(blocks))
        oracle.ref_gather([0, 0, 0], h, blocks, parts, u, u)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(len(jobs)) as ex:
        list(ex.map(work, jobs))
    transfer_s = time.perf_counter() - t0
    pressure_s, cells = _reference_pressure_time()
    return transfer_s, len(idx), pressure_s, cells


def _reference_pressure_time():
    import oracle
    from oracle.box_system import box_pressure_system, ref_blocks_for_box
    from fluidity_b200 import scenes

    n = 32
    soa, m = scenes.dam_break(n)
    x = soa[0:3].T.astype(np.float64)
    v = soa[3:6].T.astype(np.float64)
    c = soa[6:15].T.astype(np.float64)
    box = oracle.Box.make([0, 0, 0], 1.0 / n, [0, 0, 0], [n, n, n])
    fm, fq = oracle.p2g(box, x, v, c, m)
    u_pred, _ = oracle.normalize_forces(box, fm, fq, 0.0, scenes.DT, scenes.GRAVITY)
    ct = oracle.classify_cells(box, x)
    s = box_pressure_system(box, ct, u_pred)
    t0 = time.perf_counter()
    oracle.ref_project([0, 0, 0], box.h, ref_blocks_for_box(n), scenes.DT, s["cells_idx"], s["cells_val"],
                       s["faces_idx"], s["faces_kind"], s["faces_val"], tolerance_scale=1.0)
    return time.perf_counter() - t0, len(s["cells_idx"])


def cpu_baseline(soa, mass, grid, npart, ncell, budget_s=15.0, threads=1):
    sample = 400000 * threads
    res = _reference_sample_times(soa, mass, grid, sample, threads)
    if res is None:
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": "reference operators not built"}
    transfer_s, nsample, pressure_s, pcells = res
    fluid_cells = npart / 8
    step_s = transfer_s * (npart / nsample) + pressure_s * (fluid_cells / pcells)
    return {"value": round(1.0 / step_s, 8), "unit": UNIT, "cores": threads, "kind": "reference",
            "extrapolated": True, "sample": (f"DepositMac3D+GatherMac3D on {nsample} of {npart} particles ({transfer_s:.2f} s), "
                       f"ProjectMacPressure3D on its 4096-cell cap ({pcells} cells, {pressure_s:.3f} s); "
                       f"scaled linearly to the full step (pressure scaling is a lower bound)")}


def run_reference(args, world, rank):
    """The reference's own CPU operators (DepositMac3D, GatherMac3D,
    ProjectMacPressure3D compiled from its sources) on all host threads. Each
    step times a sample -- a 1/16 slice of the workload's particles split over
    the threads, plus one pressure solve at the reference's 4096-cell cap --
    and the step time is extrapolated linearly to the full workload; the line
    says so (`extrapolated`, `timed_seconds`)."""
    if rank != 0:
        return None
    import oracle
    from fluidity_b200 import scenes

    if oracle.ref() is None:
        return {"impl": "reference", "unavailable": "reference CPU operators not built (oracle/ref/Makefile)"}
    soa, mass = scenes.SCENES[args.scene](args.grid)
    npart = soa.shape[1]
    threads = max(1, os.cpu_count() or 1)
    sample = max(threads * 1000, npart // 16)
    times, timed_s, nsamples = [], 0.0, []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        res = _reference_sample_times(soa, mass, args.grid, sample, threads)
        transfer_s, nsample, pressure_s, pcells = res
        step_s = transfer_s * (npart / nsample) + pressure_s * (npart / 8 / pcells)
        if k >= args.warmup:
            times.append(step_s)
            timed_s += time.perf_counter() - t0
            nsamples.append(nsample)
    value = 1.0 / float(np.mean(times))
    desc = (f"per step: DepositMac3D+GatherMac3D on {int(np.mean(nsamples))} of {npart} particles over {threads} "
            f"threads and ProjectMacPressure3D on {pcells} cells (its 4096-cell cap), each timed and scaled "
            f"linearly to the full workload (the pressure scaling is a lower bound)")
    return {"metric": METRIC, "value": round(value, 8), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 / value, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": f"synthetic (seeded {args.scene} scene)",
            "config": dict(workload(args.scene, args.grid, args.precision), particles=npart), "impl": "reference",
            "extrapolated": True, "timed_seconds": round(timed_s, 2),
            "timed": f"{args.steps} sampled steps ({timed_s:.1f} s of host time); value extrapolated from them",
            "cpu_baseline": {"value": round(value, 8), "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": round(value, 8), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--scene", default="splash", choices=sorted(SCENES),
                    help="splash (256^3 headline) or column_drop (the 512^3 configuration)")
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1],
                    help="V-cycle storage: 1 BF16 (default, the configured mixed precision), 0 FP32")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-vs-MGPCG pressure comparison")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-column-drop", action="store_true", help="skip the 512^3 column-drop line")
    args = ap.parse_args()
    world, rank, local = _dist()
    if args.impl == "reference":
        line = run_reference(args, world, rank)
    else:
        line = run_ours(args, world, rank, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
