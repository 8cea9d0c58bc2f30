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
    p.add_argument("--requests", type=int, default=24, help="serve: number of requests")
    p.add_argument("--rates", default="5,20,80", help="serve: Poisson arrival rates (requests/s) to sweep")
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


# DRAM bytes (read + write) per step-kernel launch from the ncu captures
# summarised in profiles/ (same workload, same kernel build).
_TRAFFIC = {("fp64", 8, 16): (356.85e6, "profiles/step_kernel_uniform_swirl_l8_mx16.md"),
            ("mixed", 8, 16): (357.08e6, "profiles/step_kernel_mixed_uniform_swirl_l8_mx16.md")}


def _profiled_traffic(args):
    t = _TRAFFIC.get((args.precision, args.level, args.mx))
    if t is None or args.step_variant not in (0, 3):
        return None
    return {"bytes_per_launch": t[0], "source": t[1]}


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
    import cases

    cfg = cases.swirl_uniform(level=args.level, mx=args.mx)
    dt = cases.swirl_dt(level=args.level, mx=args.mx)
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
    import cases

    cfg = cases.swirl_uniform(level=args.level, mx=args.mx)
    dt = cases.swirl_dt(level=args.level, mx=args.mx)
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
        for _ in range(args.steps):
            s.advance_all_levels(t, dt)
            t += dt
        e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            torch.distributed.barrier()
    ms = e0.elapsed_time(e1)
    c1 = s.counters()
    launches = c1["count_kernel_launches"] - c0["count_kernel_launches"]
    cells = (c1["count_single_step"] - c0["count_single_step"]) * args.mx * args.mx
    ms_max, total_cells = replicas.aggregate(ms, cells, torch.distributed if dist else None)

    # --- step-kernel alone: K launches of the level update between events ---
    nk = max(5, args.steps)
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    k0.record(stream)
    for _ in range(nk):
        s.update_single_step_async(args.level, t, dt)
    k1.record(stream)
    torch.cuda.synchronize()
    step_ms = k0.elapsed_time(k1) / nk
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
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
                               + ("FP64 plain" if args.precision == "fp64" else "mixed FP32/FP64"),
                   "patches": npatch, "cells": cells_per_step, "l2_flush": "inputs larger than L2",
                   "parallelism": f"{world} independent replicas" if world > 1 else "single GPU",
                   "step_kernel_ms": step_ms, "ghost_fill_ms": ghost_ms},
        "clocks": clk.summary(),
        "e2e": {"value": total_cells / (e2e_ms * 1e-3),
                "unit": "cell-updates/s",
                "h2d_bytes_per_step": state_bytes / args.steps + 16,
                "d2h_bytes_per_step": state_bytes / args.steps + 8},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": _profiled_traffic(args),
                     "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback",
                     "bytes_per_cell": bytes_per_cell, "kernel": "step_kernel"},
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
# AMR shallow water: dam break, Roe solver, levels 3..6, mx = 32, subcycling,
# gradient tagging, regrid after every macro step, adaptive dt
# ----------------------------------------------------------------------------
def _amr_cfg(seed=0, workload="amr_radialdam", mx=32):
    """amr_radialdam: shallow water, levels 3-6, mx 32; amr_quadrants: Euler
    quadrants, levels 2-7, mx from --mx (8, 16, 32 or 64)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import cases

    if workload == "amr_quadrants":
        return cases.quadrants_amr(seed=seed, minlevel=2, maxlevel=7, mx=mx)
    return cases.radialdam_amr(seed=seed, minlevel=3, maxlevel=6, mx=32)


def _next_dt(dt, cfl, cfg):
    # fclaw2d_run: dt_new = dt * desired_cfl / cfl
    return dt * cfg.desired_cfl / cfl if cfl > 0 else dt


def run_amr(args, rank, world, local_rank):
    import torch

    import cases
    import forestclaw_b200 as fcb

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.current_stream()
    cfg = _amr_cfg(workload=args.workload, mx=args.mx)
    opts = cases.to_options(cfg)
    opts.precision = fcb.PRECISION_MIXED if args.precision == "mixed" else fcb.PRECISION_FP64
    opts.macro_graph = args.macro_graph
    s = fcb.Solver(opts, stream=stream.cuda_stream)
    s.initialize()
    t, dt = 0.0, cfg.initial_dt
    for _ in range(args.warmup):
        cfl = s.advance_all_levels(t, dt)
        t += dt
        s.regrid()
        dt = _next_dt(dt, cfl, cfg)
    torch.cuda.synchronize()
    c0 = s.counters()
    adv_ms, reg_s, patches = 0.0, 0.0, []
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
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
            dt = _next_dt(dt, cfl, cfg)
    c1 = s.counters()
    cells = (c1["count_single_step"] - c0["count_single_step"]) * cfg.mx * cfg.my
    if rank != 0:
        return None
    hbm, src = peaks()
    # 8*meqn*(1 + (mx+4)^2/mx^2): ghosted read + interior write
    bytes_per_cell = 8.0 * cfg.meqn * (1.0 + (cfg.mx + 4) ** 2 / cfg.mx ** 2)
    euler = args.workload == "amr_quadrants"
    achieved = cells * bytes_per_cell / (adv_ms * 1e-3) / 1e9
    line = {
        "metric": "cell-updates/s", "value": cells / (adv_ms * 1e-3), "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": adv_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32/f64", "data": "synthetic",
        "config": {"workload": (f"AMR Euler quadrants, Roe, levels 2-7, mx=my={cfg.mx}, subcycled, "
                                if euler else "AMR shallow-water dam break, Roe, levels 3-6, mx=my=32, subcycled, ")
                               + 
                               "regrid every macro step (advance phase timed; regrid reported apart)",
                   "patches_min": min(patches), "patches_max": max(patches),
                   "regrid_ms_per_step": reg_s * 1e3 / args.steps, "macro_graph": args.macro_graph,
                   "graph_replays": c1["count_graph_replays"] - c0["count_graph_replays"],
                   "launches_per_step": (c1["count_kernel_launches"] - c0["count_kernel_launches"]) / args.steps},
        "clocks": clk.summary(),
        "gpu_launches": c1["count_kernel_launches"] - c0["count_kernel_launches"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "bytes_per_cell": bytes_per_cell, "kernel": "advance phase (all kernels)",
                     "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback"},
        "roofline_fp": fp_roofline("euler4_roe_order22" if euler else "swe_roe_order22", cfg.mx,
                                   cells / (adv_ms * 1e-3), args.precision,
                                   stream.cuda_stream),
    }
    if world == 1:
        line["cpu_baseline"] = amr_cpu_sample(args.cpu_seconds, cfg)
    s.close()
    return line


def amr_cpu_sample(budget_s, cfg):
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle as O

    O.use_library(native_oracle())
    o = O.OracleSolver(cfg)
    o.initialize()
    t, dt, el, cells, n = 0.0, cfg.initial_dt, 0.0, 0, 0
    while el < budget_s and n < 50:
        c0 = o.counters()["count_single_step"]
        t0 = time.perf_counter()
        cfl = o.advance(t, dt)
        el += time.perf_counter() - t0
        cells += (o.counters()["count_single_step"] - c0) * cfg.mx * cfg.my
        t += dt
        o.regrid()
        dt = _next_dt(dt, cfl, cfg)
        n += 1
    return {"value": cells / el, "unit": "cell-updates/s", "cores": cpu_threads(), "kind": "port",
            "sample": f"first {n} macro steps of the same AMR run (advance phase, {el:.2f} s), C++ restatement "
                      f"of the reference, OpenMP over the patches of each level"}


# ----------------------------------------------------------------------------
# Shallow water over bathymetry (GeoClaw f-waves): lake at rest over a Gaussian
# bump plus a surface pulse, levels 4..7, mx = 32, subcycled, gradient tagging,
# regrid every macro step, fixed dt.  --precision mixed also reports the error
# against the same run in FP64, the mass drift and the lake-at-rest residual.
# ----------------------------------------------------------------------------
def _bathy_cfg(amp=1e-3):
    import cases

    return cases.bathy_lake(minlevel=4, maxlevel=7, mx=32, seed=0, amp=amp, width=0.05)


def _bathy_dt():
    return 0.5 / (32 * 16)  # CFL about 0.5 on level 4 (|u| + sqrt(g h) <= 1)


def _bathy_run(opts, steps, t0=0.0, stream=None, timed=False):
    """advance + regrid `steps` times; returns (solver, advance ms, cells, patch
    counts); the solver's `bench_launches` holds the launches of the advances."""
    import torch

    import forestclaw_b200 as fcb

    s = fcb.Solver(opts, stream=stream.cuda_stream if stream is not None else 0)
    s.initialize()
    t, dt, ms, cells, patches = t0, _bathy_dt(), 0.0, 0, []
    s.bench_launches = 0
    for _ in range(steps):
        c = s.counters()
        c0, l0 = c["count_single_step"], c["count_kernel_launches"]
        if timed:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        s.advance_all_levels(t, dt)
        if timed:
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        c = s.counters()
        cells += (c["count_single_step"] - c0) * opts.mx * opts.my
        s.bench_launches += c["count_kernel_launches"] - l0
        t += dt
        s.regrid()
        patches.append(s.num_patches)
    torch.cuda.synchronize()
    return s, ms, cells, patches


def run_bathy(args, rank, world, local_rank):
    import numpy as np
    import torch

    import cases
    import forestclaw_b200 as fcb

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.current_stream()
    cfg = _bathy_cfg()
    opts = cases.to_options(cfg)
    opts.precision = fcb.PRECISION_MIXED if args.precision == "mixed" else fcb.PRECISION_FP64
    opts.macro_graph = args.macro_graph
    # warm-up: the first macro steps of the same run (plans, autotuning, graph)
    w, _, _, _ = _bathy_run(opts, args.warmup, stream=stream)
    w.close()
    with ClockSampler(local_rank) as clk:
        s, ms, cells, patches = _bathy_run(opts, args.steps, stream=stream, timed=True)
    from forestclaw_b200 import replicas

    ms_max, total_cells = replicas.aggregate(ms, cells, torch.distributed if world > 1 else None)
    accuracy = None
    if args.precision == "mixed" and rank == 0:
        o64 = cases.to_options(cfg)
        o64.macro_graph = args.macro_graph
        ref, _, _, _ = _bathy_run(o64, args.steps, stream=stream)
        acc = {"against": "the same run in FP64 on the GPU", "same_mesh": ref.leaves() == s.leaves()}
        q0s = None
        if acc["same_mesh"]:
            qm, qf = s.get_q(), ref.get_q()
            m = cfg.mbc
            a, b = qm[..., m:-m, m:-m], qf[..., m:-m, m:-m]
            acc["l1_rel"] = float(np.abs(a - b).sum() / np.abs(b).sum())
            acc["max_rel"] = float(np.abs(a - b).max() / max(1.0, np.abs(b).max()))
            mm, mf = np.asarray(s.conservation_check()), np.asarray(ref.conservation_check())
            acc["mass_drift_rel"] = float(np.max(np.abs(mm - mf)) / np.max(np.abs(mf)))
        ref.close()
        # lake at rest (no pulse): the largest change of any cell after the same steps
        lake = cases.to_options(_bathy_cfg(amp=0.0))
        lake.precision = fcb.PRECISION_MIXED
        lake.macro_graph = args.macro_graph
        ls = fcb.Solver(lake, stream=stream.cuda_stream)
        ls.initialize()
        q0s = ls.get_q()
        t = 0.0
        for _ in range(args.steps):
            ls.advance_all_levels(t, _bathy_dt())
            t += _bathy_dt()
        m = cfg.mbc
        acc["lake_at_rest_max_change"] = float(np.abs(ls.get_q() - q0s)[..., m:-m, m:-m].max())
        ls.close()
        accuracy = acc
    if rank != 0:
        s.close()
        return None
    hbm, src = peaks()
    bytes_per_cell = 64.5  # meqn 3 + stored b, mx 32, mbc 2
    achieved = total_cells * bytes_per_cell / (ms_max * 1e-3) / 1e9
    line = {
        "metric": "cell-updates/s", "value": total_cells / (ms_max * 1e-3), "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32/f64", "data": "synthetic",
        "config": {"workload": "shallow water over bathymetry (GeoClaw f-waves), lake at rest + pulse 1e-3, "
                               "levels 4-7, mx=my=32, subcycled, regrid every macro step (advance phase timed)",
                   "patches_min": min(patches), "patches_max": max(patches), "macro_graph": args.macro_graph,
                   "accuracy": accuracy},
        "clocks": clk.summary(),
        "gpu_launches": s.bench_launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "bytes_per_cell": bytes_per_cell, "kernel": "advance phase (all kernels)",
                     "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback"},
        "roofline_fp": fp_roofline("geoclaw_fwave_order20", cfg.mx, total_cells / (ms_max * 1e-3), args.precision,
                                   stream.cuda_stream),
    }
    s.close()
    return line


# ----------------------------------------------------------------------------
# Ensemble serving: Poisson stream of shallow-water dam-break requests
# ----------------------------------------------------------------------------
def _serve_requests(n, seed, precision):
    """Dam breaks with radius ~ U(0.1, 0.3), inner depth ~ U(1.5, 3), outer 1,
    maxlevel ~ U{4, 5}, mx ~ {16, 32}, t_final ~ U(0.02, 0.05); levels from 2,
    non-subcycled, regrid every macro step, adaptive dt (desired CFL 0.9)."""
    import cases
    import forestclaw_b200 as fcb

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        r0, hin = rng.uniform(0.1, 0.3), rng.uniform(1.5, 3.0)
        maxlevel, mx = int(rng.integers(4, 6)), int(rng.choice([16, 32]))
        cfg = cases.radialdam_amr(seed=0, minlevel=2, maxlevel=maxlevel, mx=mx, tfinal=float(rng.uniform(0.02, 0.05)))
        cfg = cases.replace(cfg, pparams=(0.5, 0.5, r0, hin, 1.0), initial_dt=0.9 / (mx * 4) / (hin ** 0.5 + 1))
        o = cases.to_options(cfg)
        o.subcycle = 0
        o.precision = fcb.PRECISION_MIXED if precision == "mixed" else fcb.PRECISION_FP64
        out.append(o)
    return out


def run_serve(args, rank, world, local_rank):
    import torch

    from forestclaw_b200.serve import Server, poisson_stream

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.current_stream().cuda_stream
    reqs = _serve_requests(args.requests, 7 + rank, args.precision)
    budget = int(0.5 * torch.cuda.get_device_properties(local_rank).total_memory)
    # isolated latency of each request (alone on the GPU)
    iso = []
    for o in reqs:
        sv = Server(budget, stream)
        r = poisson_stream(sv, [o], rate=0.0)
        iso.append(r.latencies[0])
        sv.close()
    sweep = []
    with ClockSampler(local_rank) as clk:
        for lam in [float(x) for x in args.rates.split(",")]:
            sv = Server(budget, stream)
            r = poisson_stream(sv, reqs, rate=lam, seed=11)
            sv.close()
            sweep.append({"rate_per_s": lam, "p50_s": r.pct(50), "p99_s": r.pct(99),
                          "cell_updates_per_s": r.cell_updates / r.wall, "wall_s": r.wall,
                          "rounds": r.rounds, "launches": r.launches, "failed": r.failed,
                          "p99_over_isolated_p99": r.pct(99) / float(np.percentile(iso, 99))})
    if rank != 0:
        return None
    top = max(sweep, key=lambda d: d["cell_updates_per_s"])
    return {
        "metric": "cell-updates/s", "value": top["cell_updates_per_s"], "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.requests, "warmup": 0, "ms_per_step": top["wall_s"] * 1e3 / args.requests,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32/f64", "data": "synthetic",
        "config": {"workload": "ensemble serving: Poisson stream of shallow-water dam-break solves "
                               "(r ~ U(0.1,0.3), h_in ~ U(1.5,3), maxlevel ~ U{4,5}, mx ~ {16,32}, "
                               "t_final ~ U(0.02,0.05)), continuous batching",
                   "requests": args.requests, "isolated_p50_s": float(np.percentile(iso, 50)),
                   "isolated_p99_s": float(np.percentile(iso, 99)), "sweep": sweep},
        "p50_s": top["p50_s"], "p99_s": top["p99_s"],
        "clocks": clk.summary(),
        "gpu_launches": top["launches"],
    }


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
        run = {"amr_radialdam": run_amr, "amr_quadrants": run_amr, "bathy": run_bathy,
               "serve": run_serve}.get(args.workload, run_partitioned if args.partition else run_ours)
        line = run(args, rank, world, local_rank)
        if line:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
