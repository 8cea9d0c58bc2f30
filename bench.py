"""Benchmark of the patch hot path on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload uniform_swirl] [--level L] [--mx MX]

One "step" is one fclaw2d_advance_all_levels call (every patch updated once by
the clawpack 4.6 wave-propagation step, then the ghost-cell fill) on the
uniform swirl advection case: meqn = 1, MC limiter, order (2,2), extrapolation
boundaries, swirl velocities with T = 1, q0 = 1 for x < 0.5, FP64.  The mesh is
uniform at `level` with mx = my = 16 (level 8: 65,536 patches, 16.8 M cells).
The patch arrays (q, its pre-step copy, the time-interpolated copy and the
CFL-retry copy) take more than the 126 MB L2, so no flush is needed between
steps.

Prints ONE JSON line.  With torchrun (N > 1) each rank advances its own
replica (independent solves, weak scaling, no data-path collective); the time
is the max over ranks and the value the cell updates of all ranks over it.
With --partition the ranks share one solve instead (Morton ranges of leaves,
ghost layers exchanged through NCCL, the CFL maximum reduced every step):
strong scaling.

--impl reference times the CPU restatement of the reference's Fortran/C
(oracle/, compiled -O3 -march=native with OpenMP over the patches of a level)
on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="uniform_swirl",
                   choices=["uniform_swirl", "amr_radialdam", "amr_quadrants", "bathy", "serve"])
    p.add_argument("--requests", type=int, default=200, help="serve: number of requests")
    p.add_argument("--rates", default="auto",
                   help="serve: Poisson arrival rates (requests/s) to sweep, or auto: 0.6, 0.8 and 0.95 of the "
                        "capacity measured with every request submitted at once")
    p.add_argument("--serve-maxlevels", default="4,5,6,7", help="serve: maxlevel drawn uniformly from these")
    p.add_argument("--serve-tfinal", default="0.2,1.0", help="serve: final time ~ U(a, b)")
    p.add_argument("--serve-work-limit", type=float, default=3e6,
                   help="serve: cap on the cells of the admitted solves' meshes (0: none); without one, "
                        "concurrency and the per-solve host work of a round grow under load")
    p.add_argument("--extras", type=int, default=1,
                   help="default workload: 1 also measures the other configurations (sub-objects of the line)")
    p.add_argument("--extra-requests", type=int, default=200, help="requests of the serving sub-object (0: skip)")
    p.add_argument("--level", type=int, default=8)
    p.add_argument("--mx", type=int, default=16)
    p.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline sample budget")
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                   help="fp64: the reference's arithmetic; mixed: FP32 solves, FP64 sums and state")
    p.add_argument("--macro-graph", type=int, default=2, choices=[0, 1, 2],
                   help="1: replay each macro step from a captured CUDA graph; 0: host launches; 2: automatic")
    p.add_argument("--step-variant", type=int, default=0, help="0 library's choice, 1 CTA rows, 2 warp, 3 pipelined CTA")
    p.add_argument("--partition", action="store_true",
                   help="uniform workload: one solve partitioned over the ranks (NCCL ghost exchange, "
                        "strong scaling) instead of one replica per rank")
    return p.parse_args()


# ----------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._first = threading.Event()
        self._p = None
        self._t = None
        self._start = 0

    def _read(self):
        for line in self._p.stdout:
            parts = [x.strip() for x in line.strip().split(",")]
            if len(parts) > 2:
                self.samples.append(parts)
                self._first.set()

    def __enter__(self):
        # one long-lived nvidia-smi (NVML initialised once), its first sample
        # taken before the timed region starts
        try:
            self._p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                        "--format=csv,noheader,nounits", "-lms", "200"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._p = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        self._first.wait(5.0)
        self._start = len(self.samples)
        return self

    def __exit__(self, *a):
        if self._p is None:
            return
        self._p.terminate()
        try:
            self._p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self._p.kill()
            self._p.wait(timeout=5)
        self._t.join(timeout=5)
        if len(self.samples) > self._start:
            self.samples = self.samples[self._start:]

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        smax = max((float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 5 + k and s[5 + k].lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(self.samples)}


# DRAM bytes (read + write) per step-kernel launch, dram__bytes_read.sum +
# dram__bytes_write.sum from an ncu capture of the same kernel on the same
# workload (level 8, mx = 16), keyed by (precision, level, mx, fused step).
_TRAFFIC = {("fp64", 8, 16, False): 356.85e6, ("mixed", 8, 16, False): 357.08e6,
            ("fp64", 8, 16, True): 374.58e6}


def _profiled_traffic(args, fused):
    t = _TRAFFIC.get((args.precision, args.level, args.mx, bool(fused)))
    if t is None or args.step_variant not in (0, 3):
        return None
    return {"bytes_per_launch": t, "source": "ncu capture of this kernel on this workload "
                                             "(dram__bytes_read.sum + dram__bytes_write.sum)"}


def peaks():
    if PEAKS_FILE.exists():
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


# ----------------------------------------------------------------------------
# CPU restatement (oracle) timing: cpu_baseline and the reference arm
# ----------------------------------------------------------------------------
def native_oracle():
    """Compile the OpenMP timing build of the oracle for this host's CPU."""
    so = ROOT / "oracle" / "liboracle_native.so"
    stamp = ROOT / "oracle" / "liboracle_native.host"
    host = open("/proc/cpuinfo").read().split("model name")[1].split("\n")[0] if Path("/proc/cpuinfo").exists() else "?"
    srcs = [str(ROOT / "oracle" / f) for f in
            ("oracle_patch.cpp", "oracle_clawpatch.cpp", "oracle_amr.cpp", "oracle_capi.cpp")]
    deps = srcs + [str(p) for p in (ROOT / "oracle").glob("*.hpp")]
    stale = so.exists() and any(Path(d).stat().st_mtime > so.stat().st_mtime for d in deps)
    if not so.exists() or stale or not stamp.exists() or stamp.read_text() != host:
        cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
        subprocess.run([cxx, "-O3", "-march=native", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fopenmp",
                        "-DORC_OPENMP", "-shared", "-o", str(so), *srcs], check=True)
        stamp.write_text(host)
    return so


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def oracle_config(o):
    """The oracle's configuration of a solve given by fcb Options (the CPU
    restatement runs the same options)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle as O

    return O.Config(mx=o.mx, my=o.my, mbc=o.mbc, meqn=o.meqn, maux=o.maux, order=tuple(o.order), mcapa=o.mcapa,
                    mwaves=o.mwaves, mthlim=tuple(o.mthlim), mthbc=tuple(o.mthbc), minlevel=o.minlevel,
                    maxlevel=o.maxlevel, subcycle=o.subcycle, regrid_interval=o.regrid_interval,
                    smooth_refine=o.smooth_refine, smooth_level=o.smooth_level, criteria=o.refinement_criteria,
                    ivar=o.threshold_variable - 1, use_fixed_dt=o.use_fixed_dt, nout=o.nout,
                    init_ghostcell=o.init_ghostcell, reduce_cfl=o.reduce_cfl, solver=o.solver_kind,
                    problem=o.problem, refine_threshold=o.refine_threshold, coarsen_threshold=o.coarsen_threshold,
                    tfinal=o.tfinal, initial_dt=o.initial_dt, max_cfl=o.max_cfl, desired_cfl=o.desired_cfl,
                    grav=o.grav, gamma=o.gamma, pparams=tuple(o.problem_params), claw_version=o.claw_version,
                    drytol=o.dry_tolerance, time_sync=o.time_sync, extent=tuple(o.extent), src_term=o.src_term,
                    brick=o.brick, periodic_x=o.periodic_x, periodic_y=o.periodic_y)


def time_oracle(cfg, dt, steps, warmup):
    """Advance the oracle `warmup` + `steps` steps; returns (seconds for `steps`, cell updates)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle as O

    O.use_library(native_oracle())
    s = O.OracleSolver(cfg)
    s.initialize()
    t = 0.0
    for _ in range(warmup):
        s.advance(t, dt)
        t += dt
    c0 = s.counters()["count_single_step"]
    t0 = time.perf_counter()
    for _ in range(steps):
        s.advance(t, dt)
        t += dt
    el = time.perf_counter() - t0
    cells = (s.counters()["count_single_step"] - c0) * cfg.mx * cfg.my
    return el, cells


def cpu_sample(args, budget_s):
    from forestclaw_b200 import workloads

    cfg = oracle_config(workloads.uniform_swirl(args.level, args.mx))
    dt = workloads.swirl_dt(args.level, args.mx)
    el1, _ = time_oracle(cfg, dt, 1, 0)
    steps = max(1, int(budget_s / max(el1, 1e-3)))
    el, cells = time_oracle(cfg, dt, steps, 1)
    return {"value": cells / el, "unit": "cell-updates/s", "cores": cpu_threads(), "kind": "port",
            "sample": f"uniform swirl level {args.level}, mx={args.mx}: {steps} steps "
                      f"({cells} cell updates, {el:.2f} s) of the C++ restatement of the reference "
                      f"Fortran (reference binary not buildable: no Fortran compiler, MPI or p4est), "
                      f"OpenMP over the patches of the level"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    from forestclaw_b200 import workloads

    cfg = oracle_config(workloads.uniform_swirl(args.level, args.mx))
    dt = workloads.swirl_dt(args.level, args.mx)
    el, cells = time_oracle(cfg, dt, args.steps, args.warmup)
    v = cells / el
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"uniform swirl advection, level {args.level}, mx=my={args.mx}, FP64",
                   "patches": 4 ** args.level, "cells": 4 ** args.level * args.mx * args.mx},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cpu_threads(), "kind": "port",
                         "sample": f"full workload, {args.steps} timed steps after {args.warmup} warm-up"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    import forestclaw_b200 as fcb
    from forestclaw_b200 import replicas, workloads

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.current_stream()
    opts = workloads.uniform_swirl(args.level, args.mx)
    opts.step_variant = args.step_variant
    opts.precision = fcb.PRECISION_MIXED if args.precision == "mixed" else fcb.PRECISION_FP64
    opts.macro_graph = args.macro_graph
    dt = workloads.swirl_dt(args.level, args.mx)
    s = fcb.Solver(opts, stream=stream.cuda_stream)
    s.initialize()
    npatch = s.num_patches
    cells_per_step = npatch * args.mx * args.mx
    t = 0.0
    for _ in range(args.warmup):
        s.advance_all_levels(t, dt)
        t += dt
    dist = world > 1
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    c0 = s.counters()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        if dist:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        # every step's CFL number goes into a running maximum on the device,
        # read back once after the last step (fixed dt needs no per-step read)
        for _ in range(args.steps):
            s.advance_all_levels_async(t, dt)
            t += dt
        max_cfl = s.read_max_cfl()
        e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            torch.distributed.barrier()
    ms = e0.elapsed_time(e1)
    if not 0.0 < max_cfl <= opts.max_cfl:
        raise RuntimeError(f"CFL number {max_cfl} outside (0, max_cfl]")
    c1 = s.counters()
    launches = c1["count_kernel_launches"] - c0["count_kernel_launches"]
    cells = (c1["count_single_step"] - c0["count_single_step"]) * args.mx * args.mx
    ms_max, total_cells = replicas.aggregate(ms, cells, torch.distributed if dist else None)

    # --- the step kernel alone: the launch an advance makes (the ghost-exchange
    # fused step when the tuner chose it), K launches on scratch copies of the
    # arrays between CUDA events on the solve's stream; with the unfused form
    # the ghost fill is timed apart ---
    nk = max(5, args.steps)
    step_ms, fused = s.step_kernel_time(t, dt, nk)
    ghost_ms = None
    if not fused:
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        g0.record(stream)
        for _ in range(nk):
            s.ghost_update(args.level, args.level, t, 0)
        g1.record(stream)
        torch.cuda.synchronize()
        ghost_ms = g0.elapsed_time(g1) / nk

    # --- end to end through the C ABI with host buffers: upload the state from
    # pinned host memory, advance K steps (host dt in, CFL out each step),
    # download the result ---
    psize = opts.meqn * opts.nx * opts.ny
    host = torch.empty(npatch * psize, dtype=torch.float64, pin_memory=True)
    hv = host.numpy().reshape(npatch, opts.meqn, opts.ny, opts.nx)
    hv[...] = s.get_q()
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    t_e2e0 = time.perf_counter()
    x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    s.set_q(hv)
    for _ in range(args.steps):
        s.advance_all_levels(t, dt)
        t += dt
    s.get_q(out=hv)
    x1.record(stream)
    torch.cuda.synchronize()
    e2e_ms, _ = replicas.aggregate(x0.elapsed_time(x1), 0, torch.distributed if dist else None)
    state_bytes = npatch * psize * 8

    if rank != 0:
        return None
    hbm, src = peaks()
    nx = opts.nx
    bytes_per_cell = 8.0 * opts.meqn * (1.0 + nx * nx / (args.mx * args.mx))
    achieved = cells_per_step * bytes_per_cell / (step_ms * 1e-3) / 1e9
    line = {
        "metric": "cell-updates/s", "value": total_cells / (ms_max * 1e-3), "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32/f64",
        "data": "synthetic",
        "config": {"workload": f"uniform swirl advection, level {args.level}, mx=my={args.mx}, "
                               + ("FP64" if args.precision == "fp64" else "mixed FP32/FP64"),
                   "patches": npatch, "cells": cells_per_step, "l2_flush": "inputs larger than L2",
                   "parallelism": f"{world} independent replicas" if world > 1 else "single GPU",
                   "step_kernel_ms": step_ms, "ghost_fill_ms": ghost_ms,
                   "ghost_fill": "fused into the step (neighbour reads)" if fused else "separate launch",
                   "e2e_state_transfer": f"the whole state uploaded once and downloaded once per {args.steps} "
                                         "steps (the arrays stay resident between steps), so e2e grows "
                                         "with --steps; every e2e step reads its CFL number back",
                   "timed_steps": "fcb_advance_all_levels_async: every step's CFL number folded into a "
                                  "device maximum, read back once after the last step, inside the timed "
                                  "region",
                   "max_cfl": max_cfl},
        "clocks": clk.summary(),
        "e2e": {"value": total_cells / (e2e_ms * 1e-3),
                "unit": "cell-updates/s",
                "h2d_bytes_per_step": state_bytes / args.steps + 16,
                "d2h_bytes_per_step": state_bytes / args.steps + 8},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": _profiled_traffic(args, fused),
                     "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback",
                     "bytes_per_cell": bytes_per_cell,
                     "kernel": "step_kernel_pipe (ghost-exchange fused)" if fused else "step kernel"},
        "roofline_fp": fp_roofline("advection_swirl_order22", args.mx, cells_per_step / (step_ms * 1e-3),
                                   args.precision, stream.cuda_stream),
    }
    if args.precision == "mixed":
        line["config"]["accuracy"] = _mixed_accuracy(args, opts, dt, stream)
    if world == 1:
        sys.path.insert(0, str(ROOT / "tests"))
        line["cpu_baseline"] = cpu_sample(args, args.cpu_seconds)
    s.close()
    return line


def run_partitioned(args, rank, world, local_rank):
    """One uniform swirl solve split over the ranks (Morton ranges, NCCL
    ghost-layer exchange, global CFL maximum every step): strong scaling."""
    import torch

    import forestclaw_b200 as fcb
    from forestclaw_b200 import replicas, workloads

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.current_stream()
    uid = [fcb.nccl_unique_id() if rank == 0 else None]
    if world > 1:
        torch.distributed.broadcast_object_list(uid, src=0)
    comm = fcb.nccl_comm(uid[0], rank, world, timeout_s=120.0)
    opts = workloads.uniform_swirl(args.level, args.mx)
    opts.step_variant = args.step_variant
    opts.precision = fcb.PRECISION_MIXED if args.precision == "mixed" else fcb.PRECISION_FP64
    dt = workloads.swirl_dt(args.level, args.mx)
    s = fcb.Solver(opts, stream=stream.cuda_stream, comm=comm)
    s.initialize()
    info = s.partition_info()
    t = 0.0

    def step(t):
        return s.global_maximum(s.advance_all_levels(t, dt))

    for _ in range(args.warmup):
        step(t)
        t += dt
    torch.cuda.synchronize()
    c0 = s.counters()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step(t)
            t += dt
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
    c1 = s.counters()
    cells = (c1["count_single_step"] - c0["count_single_step"]) * args.mx * args.mx
    launches = c1["count_kernel_launches"] - c0["count_kernel_launches"]
    d = torch.distributed if world > 1 else None
    ms_max, total_cells = replicas.aggregate(e0.elapsed_time(e1), cells, d)
    # end to end: this rank's patches from pinned host memory, K steps, back to the host
    psize = opts.meqn * opts.nx * opts.ny
    npatch = s.num_patches
    host = torch.empty(npatch * psize, dtype=torch.float64, pin_memory=True)
    hv = host.numpy().reshape(npatch, opts.meqn, opts.ny, opts.nx)
    s.get_q(out=hv)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    s.set_q(hv)
    for _ in range(args.steps):
        step(t)
        t += dt
    s.get_q(out=hv)
    x1.record(stream)
    torch.cuda.synchronize()
    e2e_ms, _ = replicas.aggregate(x0.elapsed_time(x1), 0, d)
    own_bytes = info["count"] * psize * 8
    s.close()
    comm.close()
    if rank != 0:
        return None
    return {
        "metric": "cell-updates/s", "value": total_cells / (ms_max * 1e-3), "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32/f64", "data": "synthetic",
        "config": {"workload": f"uniform swirl advection, level {args.level}, mx=my={args.mx}, one solve "
                               f"partitioned over {world} rank(s)",
                   "patches": npatch, "l2_flush": "inputs larger than L2",
                   "parallelism": f"partitioned, {world} rank(s), NCCL ghost-layer exchange"},
        "clocks": clk.summary(),
        "e2e": {"value": total_cells / (e2e_ms * 1e-3), "unit": "cell-updates/s",
                "h2d_bytes_per_step": own_bytes / args.steps + 16, "d2h_bytes_per_step": own_bytes / args.steps + 8},
        "gpu_launches": launches,
    }


def _mixed_accuracy(args, opts, dt, stream, steps=20):
    """The mixed form against the FP64 form on the GPU after `steps` steps of
    the same workload: relative L1 and max-norm error of the interior cells and
    the relative difference of the mass sums."""
    import dataclasses

    import numpy as np

    import forestclaw_b200 as fcb

    q = {}
    mass = {}
    for prec in (fcb.PRECISION_MIXED, fcb.PRECISION_FP64):
        o = dataclasses.replace(opts, precision=prec)
        s = fcb.Solver(o, stream=stream.cuda_stream)
        s.initialize()
        t = 0.0
        for _ in range(steps):
            s.advance_all_levels(t, dt)
            t += dt
        q[prec] = s.get_q()
        mass[prec] = np.asarray(s.conservation_check())
        s.close()
    m = opts.mbc
    a, b = q[fcb.PRECISION_MIXED][..., m:-m, m:-m], q[fcb.PRECISION_FP64][..., m:-m, m:-m]
    return {"against": f"the FP64 form on the GPU after {steps} steps",
            "l1_rel": float(np.abs(a - b).sum() / np.abs(b).sum()),
            "max_rel": float(np.abs(a - b).max() / max(1.0, np.abs(b).max())),
            "mass_drift_rel": float(np.max(np.abs(mass[fcb.PRECISION_MIXED] - mass[fcb.PRECISION_FP64]))
                                    / np.max(np.abs(mass[fcb.PRECISION_FP64])))}


# FP64 operations per interior cell update of the reference's patch step
# (adds, multiplies, divides, square roots, compare/selects; ghost-region work
# included), counted by the instrumented build of the CPU restatement on dense
# seeded inputs: `make -C oracle flopcount && oracle/flopcount`.  Keyed by
# (case, mx); tests/test_flopcount.py checks them against that program.
FP64_OPS_PER_CELL = {
    ("advection_swirl_order22", 8): 244.5,
    ("advection_swirl_order22", 16): 193.25,
    ("advection_swirl_order22", 32): 169.875,
    ("swe_roe_order22", 16): 1244.9609,
    ("swe_roe_order22", 32): 1090.248,
    ("geoclaw_fwave_order20", 32): 1326.3662,
    ("euler4_roe_order22", 8): 2549.3125,
    ("euler4_roe_order22", 16): 2005.2109,
    ("euler4_roe_order22", 32): 1756.8027,
    ("euler4_roe_order22", 64): 1635.3647,
}


def fp_roofline(case, mx, cells_per_s, precision, stream):
    """Algorithmic FP64 operations per second of the step against this GPU's
    measured add/multiply issue rate (FP64; FP32 for the mixed form, whose
    solves run in FP32)."""
    import forestclaw_b200 as fcb

    ops = FP64_OPS_PER_CELL.get((case, mx))
    if ops is None:
        return None
    fp64 = precision == "fp64"
    peak = fcb.measure_fp_rate(fp64, stream) / 1e9
    achieved = ops * cells_per_s / 1e9
    return {"bound": "fp64 pipe" if fp64 else "fp32 pipe", "achieved": achieved, "peak": peak,
            "unit": "Gop/s", "frac": achieved / peak, "ops_per_cell": ops,
            "peak_source": "measured on this GPU (fcb_measure_fp_rate: lane add/multiply per second)"}


# ----------------------------------------------------------------------------
# AMR workloads: shallow water (levels 3-6, mx 32), Euler quadrants (levels
# 2-7), shallow water over bathymetry (levels 4-7, mx 32).  One "step" is one
# macro step (fcb_advance_all_levels) followed by a regrid; the advance phase
# is timed with CUDA events on the solve's stream, the regrid on the host clock.
# ----------------------------------------------------------------------------
def _amr_options(workload, mx, precision):
    import forestclaw_b200 as fcb
    from forestclaw_b200 import workloads

    if workload == "amr_quadrants":
        o = workloads.amr_euler(seed=0, mx=mx)
    elif workload == "bathy":
        o = workloads.bathymetry(seed=0)
    else:
        o = workloads.amr_shallow_water(seed=0)
    o.precision = fcb.PRECISION_MIXED if precision == "mixed" else fcb.PRECISION_FP64
    return o


def _next_dt(dt, cfl, o):
    # fclaw2d_run: dt_new = dt * desired_cfl / cfl (fixed dt when use_fixed_dt)
    if o.use_fixed_dt:
        return dt
    return dt * o.desired_cfl / cfl if cfl > 0 else dt


def _first_dt(o):
    from forestclaw_b200 import workloads

    return workloads.bathymetry_dt(o.minlevel, o.mx) if o.problem == 3 else o.initial_dt


def amr_measure(opts, steps, warmup, stream, local_rank, keep=False):
    """Warm-up macro steps (plans, tuned forms, the macro-step graph), then
    `steps` timed ones; every macro step is followed by a regrid."""
    import torch

    import forestclaw_b200 as fcb

    s = fcb.Solver(opts, stream=stream.cuda_stream)
    s.initialize()
    t, dt = 0.0, _first_dt(opts)
    for _ in range(warmup):
        cfl = s.advance_all_levels(t, dt)
        t += dt
        s.regrid()
        dt = _next_dt(dt, cfl, opts)
    torch.cuda.synchronize()
    c0 = s.counters()
    adv_ms, reg_s, patches = 0.0, 0.0, []
    with ClockSampler(local_rank) as clk:
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            cfl = s.advance_all_levels(t, dt)
            e1.record(stream)
            torch.cuda.synchronize()
            adv_ms += e0.elapsed_time(e1)
            t += dt
            r0 = time.perf_counter()
            s.regrid()
            torch.cuda.synchronize()
            reg_s += time.perf_counter() - r0
            patches.append(s.num_patches)
            dt = _next_dt(dt, cfl, opts)
    c1 = s.counters()
    cells = (c1["count_single_step"] - c0["count_single_step"]) * opts.mx * opts.my
    out = {"value": cells / (adv_ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": adv_ms / steps,
           "steps": steps, "warmup": warmup, "cell_updates": cells,
           "patches_min": min(patches), "patches_max": max(patches),
           "regrid_ms_per_step": reg_s * 1e3 / steps,
           "graph_replays": c1["count_graph_replays"] - c0["count_graph_replays"],
           "gpu_launches": c1["count_kernel_launches"] - c0["count_kernel_launches"],
           "clocks": clk.summary()}
    if keep:
        out["solver"] = s
    else:
        s.close()
    return out


def _fp_case(opts):
    return {1: "swe_roe_order22", 2: "euler4_roe_order22", 3: "geoclaw_fwave_order20",
            0: "advection_swirl_order22"}[opts.solver_kind]


def _bytes_per_cell(opts):
    # ghosted read + interior write of the state, plus the stored aux read
    # (bathymetry; capacity and edge velocities of the manifold solver)
    r = (opts.mx + 2 * opts.mbc) ** 2 / (opts.mx * opts.my)
    aux = opts.maux if opts.solver_kind in (3, 4) else 0
    return 8.0 * (opts.meqn * (1.0 + r) + aux * r)


def run_amr(args, rank, world, local_rank):
    import torch

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.current_stream()
    opts = _amr_options(args.workload, args.mx, args.precision)
    opts.macro_graph = args.macro_graph
    m = amr_measure(opts, args.steps, args.warmup, stream, local_rank)
    if rank != 0:
        return None
    hbm, src = peaks()
    bpc = _bytes_per_cell(opts)
    achieved = m["value"] * bpc / 1e9
    name = {"amr_quadrants": f"AMR Euler quadrants, Roe, levels 2-7, mx=my={opts.mx}, subcycled",
            "bathy": "shallow water over bathymetry (GeoClaw f-waves), lake at rest + pulse 1e-3, levels 4-7, "
                     "mx=my=32, subcycled",
            }.get(args.workload, "AMR shallow-water dam break, Roe, levels 3-6, mx=my=32, subcycled")
    line = {
        "metric": "cell-updates/s", "value": m["value"], "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32/f64", "data": "synthetic",
        "config": {"workload": name + ", regrid every macro step (advance phase timed; regrid reported apart)",
                   "patches_min": m["patches_min"], "patches_max": m["patches_max"],
                   "regrid_ms_per_step": m["regrid_ms_per_step"], "macro_graph": args.macro_graph,
                   "graph_replays": m["graph_replays"]},
        "clocks": m["clocks"],
        "gpu_launches": m["gpu_launches"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "bytes_per_cell": bpc, "kernel": "advance phase (all kernels)",
                     "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback"},
        "roofline_fp": fp_roofline(_fp_case(opts), opts.mx, m["value"], args.precision, stream.cuda_stream),
    }
    if args.workload == "bathy" and args.precision == "mixed":
        line["config"]["accuracy"] = bathy_accuracy(args.steps, args.macro_graph, stream)
    if world == 1:
        line["cpu_baseline"] = amr_cpu_sample(args.cpu_seconds, opts)
    return line


def amr_cpu_sample(budget_s, opts):
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle as O

    O.use_library(native_oracle())
    cfg = oracle_config(opts)
    o = O.OracleSolver(cfg)
    o.initialize()
    t, dt, el, cells, n = 0.0, _first_dt(opts), 0.0, 0, 0
    while el < budget_s and n < 50:
        c0 = o.counters()["count_single_step"]
        t0 = time.perf_counter()
        cfl = o.advance(t, dt)
        el += time.perf_counter() - t0
        cells += (o.counters()["count_single_step"] - c0) * cfg.mx * cfg.my
        t += dt
        o.regrid()
        dt = _next_dt(dt, cfl, opts)
        n += 1
    return {"value": cells / el, "unit": "cell-updates/s", "cores": cpu_threads(), "kind": "port",
            "sample": f"first {n} macro steps of the same AMR run (advance phase, {el:.2f} s), C++ restatement "
                      f"of the reference, OpenMP over the patches of each level"}


def bathy_accuracy(steps, macro_graph, stream):
    """The mixed form of the bathymetry run against the same run in FP64 after
    `steps` macro steps with regrids: relative L1 and max error of the interior
    cells, mass drift, and the lake at rest (no pulse) after the same steps."""
    import forestclaw_b200 as fcb
    from forestclaw_b200 import workloads

    def run(o):
        s = fcb.Solver(o, stream=stream.cuda_stream)
        s.initialize()
        t, dt = 0.0, workloads.bathymetry_dt(o.minlevel, o.mx)
        for _ in range(steps):
            s.advance_all_levels(t, dt)
            t += dt
            if o.regrid_interval:
                s.regrid()
        return s

    res = {}
    for prec in (fcb.PRECISION_MIXED, fcb.PRECISION_FP64):
        o = workloads.bathymetry(seed=0)
        o.precision, o.macro_graph = prec, macro_graph
        res[prec] = run(o)
    sm, sf = res[fcb.PRECISION_MIXED], res[fcb.PRECISION_FP64]
    acc = {"against": f"the same run in FP64 on the GPU after {steps} macro steps with regrids",
           "same_mesh": sm.leaves() == sf.leaves()}
    if acc["same_mesh"]:
        qm, qf = sm.get_q(), sf.get_q()
        a, b = qm[..., 2:-2, 2:-2], qf[..., 2:-2, 2:-2]
        acc["l1_rel"] = float(np.abs(a - b).sum() / np.abs(b).sum())
        acc["max_rel"] = float(np.abs(a - b).max() / max(1.0, np.abs(b).max()))
        mm, mf = np.asarray(sm.conservation_check()), np.asarray(sf.conservation_check())
        acc["mass_drift_rel"] = float(np.max(np.abs(mm - mf)) / np.max(np.abs(mf)))
    sm.close()
    sf.close()
    lake = workloads.bathymetry(seed=0, amp=0.0)
    lake.precision, lake.macro_graph, lake.regrid_interval = fcb.PRECISION_MIXED, macro_graph, 0
    ls = fcb.Solver(lake, stream=stream.cuda_stream)
    ls.initialize()
    q0 = ls.get_q()
    t, dt = 0.0, workloads.bathymetry_dt(lake.minlevel, lake.mx)
    for _ in range(steps):
        ls.advance_all_levels(t, dt)
        t += dt
    acc["lake_at_rest_max_change"] = float(np.abs(ls.get_q() - q0)[..., 2:-2, 2:-2].max())
    ls.close()
    return acc


# ----------------------------------------------------------------------------
# Ensemble serving: Poisson stream of shallow-water dam-break requests
# ----------------------------------------------------------------------------
def serve_measure(requests, rates, local_rank, stream, label, work_limit=0, loads=(0.6, 0.8, 0.95)):
    """Isolated latency and cell updates of every request (alone on the GPU,
    after one untimed solve that loads the kernels and fills the autotuner's
    and the memory pool's caches); the saturation throughput (every request
    submitted at once); then Poisson streams: at the given rates, or, with
    rates None, at the given fractions of the capacity the saturation run
    implies (requests/s = saturation cell-updates/s over the mean cell updates
    of a request).  Each point reports p50/p99 latency and the aggregate
    cell-updates/s; the knee is the lowest rate whose throughput is within 5 %
    of the best point's."""
    import torch

    from forestclaw_b200.serve import Server, poisson_stream

    budget = int(0.5 * torch.cuda.get_device_properties(local_rank).total_memory)
    sv = Server(budget, stream)
    poisson_stream(sv, requests[:1], rate=0.0)
    sv.close()
    iso, work = [], 0
    for o in requests:
        sv = Server(budget, stream)
        r = poisson_stream(sv, [o], rate=0.0)
        iso.append(r.latencies[0])
        work += r.cell_updates
        sv.close()
    iso_p99 = float(np.percentile(iso, 99))
    sweep = []
    with ClockSampler(local_rank) as clk:
        sv = Server(budget, stream)
        sv.set_work_limit(work_limit)
        r = poisson_stream(sv, requests, rate=0.0)
        sv.close()
        sat = r.cell_updates / r.wall
        capacity = len(requests) * sat / work
        points = [(lam, None) for lam in rates] if rates else [(f * capacity, f) for f in loads]
        for lam, f in points:
            sv = Server(budget, stream)
            sv.set_work_limit(work_limit)
            r = poisson_stream(sv, requests, rate=lam, seed=11)
            sv.close()
            sweep.append({"rate_per_s": lam, "load": f, "p50_s": r.pct(50), "p99_s": r.pct(99),
                          "cell_updates_per_s": r.cell_updates / r.wall,
                          "throughput_over_saturation": r.cell_updates / r.wall / sat, "wall_s": r.wall,
                          "rounds": r.rounds, "launches": r.launches, "failed": r.failed,
                          "p99_over_isolated_p99": r.pct(99) / iso_p99})
    top = max(sweep, key=lambda d: d["cell_updates_per_s"])
    knee = min((d for d in sweep if d["cell_updates_per_s"] >= 0.95 * top["cell_updates_per_s"]),
               key=lambda d: d["rate_per_s"])
    return {"workload": label, "requests": len(requests), "work_limit_cells": work_limit,
            "isolated_p50_s": float(np.percentile(iso, 50)), "isolated_p99_s": iso_p99,
            "saturation_cell_updates_per_s": sat, "capacity_requests_per_s": capacity, "sweep": sweep,
            "best": top, "knee": knee, "clocks": clk.summary()}


def _rates(args):
    return None if args.rates == "auto" else [float(x) for x in args.rates.split(",")]


def run_serve(args, rank, world, local_rank):
    import torch

    import forestclaw_b200 as fcb
    from forestclaw_b200 import workloads

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.current_stream().cuda_stream
    maxlevels = tuple(int(v) for v in args.serve_maxlevels.split(","))
    tf = tuple(float(v) for v in args.serve_tfinal.split(","))
    reqs = workloads.dam_break_requests(args.requests, 7 + rank, maxlevels=maxlevels, tfinal=tf)
    for o in reqs:
        o.precision = fcb.PRECISION_MIXED if args.precision == "mixed" else fcb.PRECISION_FP64
    label = (f"ensemble serving: Poisson stream of shallow-water dam-break solves (r ~ U(0.1,0.3), h_in ~ "
             f"U(1.5,3), maxlevel ~ U{{{','.join(map(str, maxlevels))}}}, mx ~ {{16,32}}, levels from 2, subcycled, "
             f"t_final ~ U({tf[0]},{tf[1]})), continuous batching")
    m = serve_measure(reqs, _rates(args), local_rank, stream, label, int(args.serve_work_limit))
    if rank != 0:
        return None
    top = m["best"]
    return {
        "metric": "cell-updates/s", "value": top["cell_updates_per_s"], "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.requests, "warmup": 0, "ms_per_step": top["wall_s"] * 1e3 / args.requests,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32/f64", "data": "synthetic",
        "config": {"workload": label, "requests": args.requests, "work_limit_cells": m["work_limit_cells"],
                   "isolated_p50_s": m["isolated_p50_s"], "isolated_p99_s": m["isolated_p99_s"],
                   "saturation_cell_updates_per_s": m["saturation_cell_updates_per_s"],
                   "capacity_requests_per_s": m["capacity_requests_per_s"], "sweep": m["sweep"], "knee": m["knee"]},
        "p50_s": top["p50_s"], "p99_s": top["p99_s"],
        "clocks": m["clocks"],
        "gpu_launches": top["launches"],
    }


# ----------------------------------------------------------------------------
# The other forms and configurations, measured in the default run and reported
# as sub-objects of its line (each with its own clocks and CUDA-event times)
# ----------------------------------------------------------------------------
def _uniform_quick(level, mx, precision, steps, warmup, stream, local_rank):
    import torch

    import forestclaw_b200 as fcb
    from forestclaw_b200 import workloads

    o = workloads.uniform_swirl(level, mx)
    o.precision = fcb.PRECISION_MIXED if precision == "mixed" else fcb.PRECISION_FP64
    dt = workloads.swirl_dt(level, mx)
    s = fcb.Solver(o, stream=stream.cuda_stream)
    s.initialize()
    t = 0.0
    for _ in range(warmup):
        s.advance_all_levels(t, dt)
        t += dt
    c0 = s.counters()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        for _ in range(steps):
            s.advance_all_levels_async(t, dt)
            t += dt
        s.read_max_cfl()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    c1 = s.counters()
    cells = (c1["count_single_step"] - c0["count_single_step"]) * mx * mx
    kms, fused = s.step_kernel_time(t, dt, max(5, steps))
    s.close()
    return {"value": cells / (ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": ms / steps, "steps": steps,
            "warmup": warmup, "step_kernel_ms": kms, "ghost_fill_fused": fused,
            "gpu_launches": c1["count_kernel_launches"] - c0["count_kernel_launches"], "clocks": clk.summary()}


def run_extras(args, local_rank, main_line):
    """Sub-objects of the default line: the mixed form of the uniform case,
    AMR shallow water (FP64, mixed), AMR Euler, bathymetry (FP64, mixed, with
    the error of the mixed form) and a serving sweep."""
    import torch

    import forestclaw_b200 as fcb
    from forestclaw_b200 import workloads

    stream = torch.cuda.current_stream()
    out = {}

    def guarded(name, fn):
        t0 = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as e:  # noqa: BLE001 - reported in the line, the main number stands
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = time.perf_counter() - t0

    def mixed_uniform():
        m = _uniform_quick(args.level, args.mx, "mixed", args.steps, args.warmup, stream, local_rank)
        m["workload"] = f"uniform swirl advection, level {args.level}, mx=my={args.mx}, mixed FP32/FP64"
        m["speedup_over_fp64"] = main_line["ms_per_step"] / m["ms_per_step"]
        m["step_kernel_speedup_over_fp64"] = main_line["config"]["step_kernel_ms"] / m["step_kernel_ms"]
        m["accuracy"] = _mixed_accuracy(args, workloads.uniform_swirl(args.level, args.mx),
                                        workloads.swirl_dt(args.level, args.mx), stream)
        m["roofline_fp"] = fp_roofline("advection_swirl_order22", args.mx, m["value"], "mixed", stream.cuda_stream)
        return m

    def amr(workload, precision, steps, mx=32):
        o = _amr_options(workload, mx, precision)
        m = amr_measure(o, steps, 2, stream, local_rank)
        m["roofline_fp"] = fp_roofline(_fp_case(o), o.mx, m["value"], precision, stream.cuda_stream)
        m["hbm_frac"] = m["value"] * _bytes_per_cell(o) / 1e9 / peaks()[0]
        return m

    def pair(workload, steps, mx=32):
        f = amr(workload, "fp64", steps, mx)
        mm = amr(workload, "mixed", steps, mx)
        return {"fp64": f, "mixed": mm, "mixed_over_fp64": mm["value"] / f["value"]}

    guarded("mixed_uniform", mixed_uniform)

    def c2():
        r = pair("amr_radialdam", 5)
        r["workload"] = ("AMR shallow-water dam break (Roe), levels 3-6, mx=my=32, subcycled, regrid every macro "
                         "step; advance phase timed, seed 0")
        return r

    guarded("amr_shallow_water", c2)

    def c3():
        r = amr("amr_quadrants", "fp64", 3, mx=16)
        r["workload"] = ("AMR Euler quadrants (Roe), levels 2-7, mx=my=16, subcycled (32 fine steps per macro "
                         "step), regrid every macro step; advance phase timed, seed 0")
        return r

    guarded("amr_euler", c3)

    def c4():
        r = pair("bathy", 3)
        r["workload"] = ("shallow water over bathymetry (GeoClaw f-waves), lake at rest + pulse 1e-3, levels 4-7, "
                         "mx=my=32, subcycled, regrid every macro step; advance phase timed")
        r["mixed_accuracy"] = bathy_accuracy(3, 2, stream)
        return r

    guarded("bathymetry", c4)

    def mapped():
        o = workloads.filament()
        m = amr_measure(o, 3, 2, stream, local_rank)
        m["hbm_frac"] = m["value"] * _bytes_per_cell(o) / 1e9 / peaks()[0]
        m["workload"] = ("filament (advection/2d/filament example 1 setup): cart-mapped 2 x 2 brick with capacity "
                         "aux(1) and psi edge velocities aux(2:3), manifold advection solver (capacity form of the "
                         "four-barrier step), levels 4-6 of each block, mx=my=32, subcycled, regrid every macro "
                         "step; advance phase timed, FP64")
        return m

    guarded("filament", mapped)

    def serving():
        reqs = workloads.dam_break_requests(args.extra_requests, 7, maxlevels=(4, 5, 6, 7), tfinal=(0.02, 0.1))
        label = ("ensemble serving, FP64: Poisson stream of shallow-water dam-break solves (r ~ U(0.1,0.3), "
                 "h_in ~ U(1.5,3), maxlevel ~ U{4..7}, mx ~ {16,32}, levels from 2, subcycled, t_final ~ "
                 "U(0.02,0.1): the configured final times scaled by 1/10 so the sweep fits the default run), "
                 "continuous batching")
        return serve_measure(reqs, _rates(args), local_rank, stream.cuda_stream, label,
                             int(args.serve_work_limit))

    if args.extra_requests > 0:
        guarded("serving", serving)
    return out


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        sys.path.insert(0, str(ROOT / "tests"))
        line = run_reference(args, rank, world)
        if line:
            print(json.dumps(line), flush=True)
        return
    import torch

    if world > 1:
        import datetime

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local_rank))
    try:
        sys.path.insert(0, str(ROOT / "tests"))
        run = {"amr_radialdam": run_amr, "amr_quadrants": run_amr, "bathy": run_amr,
               "serve": run_serve}.get(args.workload, run_partitioned if args.partition else run_ours)
        line = run(args, rank, world, local_rank)
        if line and run is run_ours and args.extras and world == 1 and args.precision == "fp64":
            line["extras"] = run_extras(args, local_rank, line)
        if line:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
