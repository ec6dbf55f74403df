"""Benchmark: relative 5D capture-tube solve (ENO2 / Lax-Friedrichs / RK2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the 89M-cell table): RelativeGrid(65, 48, 21, 21, 8.0) — 65 x 65
relative positions on [-8, 8] m, 48 headings, 21 x 21 speed levels —
reversible_free_a3 physics (both accelerations 3 m/s^2), CFL 0.8, horizon
3.0 s in 0.1-s frames = 900 RK2 steps = 1800 stage launches (the step
sequence of the reference driver, native_relative.cpp:173-190).  Values and local arithmetic are
float32 (the fast path).  One bench step = one full solve to the horizon:
initialise the capture field, advance 900 steps.

Metric: cell-backups/s = cells x stages / seconds (one cell-backup = one ENO/LF
stage update of one cell).  `value` times device-resident solves with CUDA
events on the solver's stream; `e2e` times the same solve through the public
RelativeSolver API with host buffers: the initial field uploaded from pinned
memory and the final field and arrival times read back every step.  The
field (357.7 MB) is larger than the 126 MB L2, so no flush is needed between
iterations.

Multi-GPU (torchrun): by default the N ranks solve ONE table, each owning a
range of pursuer-speed (vP) slabs, with NCCL halo exchanges after every stage
(strong scaling: `value` = the table's cell-backups over the slowest rank's
device time); `--mode replicas` gives every rank its own table instead (weak
scaling, no data-path collective).

--impl reference runs the reference's own CPU implementation of the path
(native_relative.cpp compiled from the reference sources into
oracle/_ref/relative5d) on all host cores, on a bounded sample of the same
workload (the same grid and physics, a few RK2 steps per bench step).
"""

from __future__ import annotations

import argparse
import json
import os
from pathlib import Path
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "pursuit-evasion-core_b200"))
sys.path.insert(0, str(REPO))

GRID = dict(positions=65, headings=48, p_speeds=21, e_speeds=21, extent=8.0)
HORIZON = 3.0
OUTPUT_DT = 0.1  # frame boundaries split the steps as in the reference driver
METRIC = "cell-backups/s"
REF_EXE = REPO / "oracle" / "_ref" / "relative5d"
ORACLE_LIB = REPO / "oracle" / "_build" / "liboracle.so"


def a3_config():
    from pursuit_evasion_b200.reversible.model import ReversibleConfig, VehicleLimits

    return ReversibleConfig(
        name="reversible_free_a3",
        pursuer=VehicleLimits(-1.0, 2.0, 3.0, 1.0),
        evader=VehicleLimits(-0.5, 1.0, 3.0, 2.0),
    )


def workload_name():
    g = GRID
    return (f"relative5d_eno2_lf_rk2 RelativeGrid({g['positions']},{g['headings']},"
            f"{g['p_speeds']},{g['e_speeds']},{g['extent']}) reversible_free_a3 "
            f"horizon {HORIZON} s cfl 0.8")


def bench_config(cells):
    """The `config` object of both arms' JSON lines (the same workload)."""
    return {"workload": workload_name(), "cells": cells,
            "unit_of_work": "one ENO2/LF RK2 stage update of one cell (cell-backup)",
            "l2": "inputs larger than L2 (357.7 MB field), no flush"}


# ---------------------------------------------------------------------------
# clocks during the timed region
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        fd, self.path = tempfile.mkstemp(prefix="pe_clocks_", suffix=".csv")
        os.close(fd)
        self.file = open(self.path, "w")
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.gpu_index), f"--query-gpu={self.QUERY}",
             "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=self.file, stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.close()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        sm_max = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": sm_max, "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(values, world, device="cuda"):
    """Element-wise maximum of per-rank timings (all ranks take this step)."""
    import torch

    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.tolist()


def measured_peaks():
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """dram bytes per stage launch from the committed ncu summary, if any."""
    path = REPO / "profiles" / "relative5d_stage_traffic.json"
    if path.exists():
        return json.loads(path.read_text())
    return None


# reversible_free_a3 (configs/reversible_free_a3.json of the reference) as
# plain numbers: the reference arm must not load this package.
A3_LIMITS = {
    "pursuer": dict(speed_min=-1.0, speed_max=2.0, acceleration=3.0, max_curvature=1.0),
    "evader": dict(speed_min=-0.5, speed_max=1.0, acceleration=3.0, max_curvature=2.0),
    "capture_radius": 0.3,
}


def reference_cfl_dt(cfl=0.8):
    """The CFL step limit of native_relative.cpp:76-81 for the bench grid,
    restated in plain Python so that the reference arm imports nothing from
    this package."""
    import math

    p, e = A3_LIMITS["pursuer"], A3_LIMITS["evader"]
    g = GRID
    dx = 2 * g["extent"] / (g["positions"] - 1)
    dphi = 2 * math.pi / g["headings"]
    dvp = (p["speed_max"] - p["speed_min"]) / (g["p_speeds"] - 1)
    dve = (e["speed_max"] - e["speed_min"]) / (g["e_speeds"] - 1)
    VP = max(abs(p["speed_min"]), abs(p["speed_max"]))
    VE = max(abs(e["speed_min"]), abs(e["speed_max"]))
    kp, ke = p["max_curvature"], e["max_curvature"]
    total = ((VP + VE + VP * kp * g["extent"]) / dx + (VE + VP * kp * g["extent"]) / dx
             + (VP * kp + VE * ke) / dphi + p["acceleration"] / dvp
             + e["acceleration"] / dve)
    return cfl / total


def reference_sample(steps, threads):
    """Run the reference executable (native_relative.cpp built from the
    reference sources) on the bench grid for `steps` RK2 steps; returns
    (update_seconds, internal_steps) from its own timing.json."""
    horizon = steps * reference_cfl_dt()
    p, e = A3_LIMITS["pursuer"], A3_LIMITS["evader"]
    g = GRID
    out = Path(tempfile.mkdtemp(prefix="pe_refbench_"))
    options = {
        "positions": g["positions"], "headings": g["headings"],
        "p-speeds": g["p_speeds"], "e-speeds": g["e_speeds"],
        "extent": g["extent"], "radius": A3_LIMITS["capture_radius"],
        "p-min": p["speed_min"], "p-max": p["speed_max"], "e-min": e["speed_min"],
        "e-max": e["speed_max"], "p-acceleration": p["acceleration"],
        "e-acceleration": e["acceleration"], "p-curvature": p["max_curvature"],
        "e-curvature": e["max_curvature"], "horizon": repr(horizon),
        "output-dt": repr(horizon), "order": 2, "cfl": 0.8, "threads": threads,
        "history": 0, "output": str(out),
    }
    cmd = [str(REF_EXE)] + [str(x) for k, v in options.items()
                            for x in ("--" + k, v)]
    try:
        subprocess.run(cmd, check=True, capture_output=True)
        timing = json.loads((out / "timing.json").read_text())
    finally:
        shutil.rmtree(out, ignore_errors=True)
    return float(timing["update_seconds"]), int(timing["internal_steps"])


def oracle_sample(steps, threads):
    """The oracle port (oracle/relative5d.c) on the bench grid, `steps` RK2
    steps; used only when the reference executable is not built.  Like
    reference_sample it imports nothing from this package."""
    import ctypes
    from types import SimpleNamespace

    from tests import oracle_lib

    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    o = oracle_lib.load()
    config = SimpleNamespace(pursuer=SimpleNamespace(**A3_LIMITS["pursuer"]),
                             evader=SimpleNamespace(**A3_LIMITS["evader"]),
                             capture_radius=A3_LIMITS["capture_radius"])
    cfg = o.rel_cfg(config, SimpleNamespace(**GRID))
    n = int(np.prod([GRID[k] for k in ("p_speeds", "e_speeds", "headings")])
            * GRID["positions"] ** 2)
    a = np.empty(n, np.float32)
    b = np.empty(n, np.float32)
    arr = np.empty(n, np.float32)
    o.lib.po_rel_init(ctypes.addressof(cfg), a.ctypes.data, arr.ctypes.data)
    dt = o.rel_cfl_limit(cfg)
    t0 = time.perf_counter()
    for k in range(steps):
        o.rel_stage_f32(cfg, a, b, arr, dt, k * dt, 0)
        o.rel_stage_f32(cfg, b, a, arr, dt, k * dt, 1)
    return time.perf_counter() - t0, steps


def cpu_baseline(steps=3):
    threads = os.cpu_count() or 1
    cells = int(np.prod([GRID["p_speeds"], GRID["e_speeds"], GRID["headings"],
                         GRID["positions"], GRID["positions"]]))
    if REF_EXE.exists():
        seconds, taken = reference_sample(steps, threads)
        kind = "reference"
        what = "native_relative.cpp built from the reference sources"
    else:
        seconds, taken = oracle_sample(steps, threads)
        kind = "port"
        what = "oracle/relative5d.c restatement"
    value = cells * taken * 2 / seconds
    return {
        "value": value, "unit": METRIC, "cores": threads, "kind": kind,
        "sample": (f"{what}: {taken} RK2 steps ({2 * taken} stages) of the "
                   f"{cells}-cell bench grid, update loop only, "
                   f"{seconds:.3f} s on {threads} threads"),
    }


# ---------------------------------------------------------------------------
def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    steps_per_sample = 2
    threads = os.cpu_count() or 1
    cells = int(np.prod(list(GRID.values())[:4]) * GRID["positions"])
    for _ in range(args.warmup):
        if REF_EXE.exists():
            reference_sample(steps_per_sample, threads)
        else:
            oracle_sample(steps_per_sample, threads)
    total_s = 0.0
    total_steps = 0
    for _ in range(args.steps):
        if REF_EXE.exists():
            s, n = reference_sample(steps_per_sample, threads)
        else:
            s, n = oracle_sample(steps_per_sample, threads)
        total_s += s
        total_steps += n
    value = cells * total_steps * 2 / total_s
    kind = "reference" if REF_EXE.exists() else "port"
    line = {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 storage, f64 local", "data": "synthetic (deterministic grid)",
        "config": bench_config(cells),
        "run": {"stages_per_step": 2 * steps_per_sample,
                "sample": (f"each bench step runs {steps_per_sample} RK2 steps of the same "
                           "grid and physics; the metric is per cell-stage, so it compares "
                           "with the full solve of the other arm"),
                "parallelism": f"OpenMP {threads} threads"},
        "cpu_baseline": {
            "value": value, "unit": METRIC, "cores": threads, "kind": kind,
            "sample": (f"{steps_per_sample} RK2 steps of the bench grid per "
                       f"step, update loop only (reference timing.json)"),
        },
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _timing_stream():
    """The current torch stream when it is a created one; else a new stream
    made current.  The solver handles read stream 0 as their own stream, so
    events recorded on the legacy default stream would not bracket their
    kernels."""
    import torch

    stream = torch.cuda.current_stream()
    if stream.cuda_stream == 0:
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
    return stream


def _world8d_run(grid, steps, fast):
    import torch
    from pursuit_evasion_b200.reversible.world_dp import WorldSolver

    with WorldSolver(a3_config(), grid, avoid=False, fast=fast) as s:
        stream = _timing_stream()
        s.set_stream(stream.cuda_stream)
        s.init_contact((0.5, 0.3), (0.5, 0.3))
        for _ in range(3):
            s.step(s.dt_limit)
        s.init_contact((0.5, 0.3), (0.5, 0.3))
        s.synchronize()
        s.profile(True)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(steps):
            s.step(s.dt_limit)
        t1.record(stream)
        s.synchronize()
        ms = t0.elapsed_time(t1)
        kms, _ = s.kernel_time()
        s.profile(False)
        return ms, kms, s.residual()


def world8d_section(steps=200):
    """The 8D contact game step (config 4): 11^4 positions, 9^2 headings, 7^2
    speeds (58,110,129 cells), a3 limits, 0.5 x 0.3 m footprints, CFL 0.8,
    `steps` RK2 steps from the rectangle-contact field; device time of the
    fast stage, with the reference-order (bit-exact) stage beside it."""
    from pursuit_evasion_b200.reversible.world_dp import WorldGrid

    grid = WorldGrid(11, 9, 7, 7, 3.0)
    ms, kms, residual = _world8d_run(grid, steps, fast=True)
    ms_exact, _, _ = _world8d_run(grid, steps, fast=False)
    cells = grid.states
    peak, _ = measured_peaks()
    achieved = (8 * cells + 12 * cells) * steps / (kms / 1e3) / 1e9
    return {"workload": "world8d_contact WorldGrid(11,9,7,7,3.0) a3, 0.5x0.3 m bodies, "
                        f"CFL 0.8, {steps} RK2 steps, float32 (reciprocal spacings, FMA)",
            "cells": cells, "value": cells * 2 * steps / (ms / 1e3),
            "unit": METRIC, "ms_per_rk2_step": ms / steps,
            "exact_order_ms_per_rk2_step": ms_exact / steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "algorithmic_bytes_per_rk2_step": 20 * cells},
            "last_residual": residual}


def fp64_section(float32_table):
    """The error of the float32 tables at the 3.0 s horizon against FP64
    storage on the 89M-cell grid, on the 1/8-subsampled tile (every 8th x,
    y and psi node, all speeds): the FP64-storage solve (the FP64 oracle's
    stage on the GPU, bit-identical to it) to the same horizon, the bench's
    own float32-local table (`float32_table`), and the exact path (float32
    storage, double local arithmetic: the reference's arithmetic and the
    default of free_dp.solve), whose device time is reported too."""
    import torch
    from pursuit_evasion_b200.reversible.fp64_table import RelativeSolverF64, subsampled_error
    from pursuit_evasion_b200.reversible.free_dp import RelativeGrid, output_times
    from pursuit_evasion_b200.reversible.relative_solver import RelativeSolver

    grid = RelativeGrid(**GRID)
    goals = output_times(HORIZON, OUTPUT_DT)[1:]
    stream = _timing_stream()

    def timed_solve(solver):
        solver.set_stream(stream.cuda_stream)
        solver.initialize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for goal in goals:
            solver.advance(goal)
        t1.record(stream)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1), solver.steps, solver.field()

    with RelativeSolverF64(a3_config(), grid) as r:
        ms64, steps64, reference = timed_solve(r)
    with RelativeSolver(a3_config(), grid, local_precision="float64") as s:
        ms_exact, steps, exact = timed_solve(s)
    cells = grid.states
    fast = np.asarray(float32_table).reshape(grid.shape)
    return {
        "workload": f"RelativeGrid(65,48,21,21,8.0) reversible_free_a3, CFL 0.8, {HORIZON} s = "
                    f"{steps} RK2 steps; errors on every 8th x, y, psi node and all speeds",
        "target_max_abs": 1e-4,
        "float32_local_vs_fp64": subsampled_error(fast, reference, 8),
        "exact_path_vs_fp64": subsampled_error(exact, reference, 8),
        "exact_path": {"value": cells * 2 * steps / (ms_exact / 1e3), "unit": METRIC,
                       "ms_per_rk2_step": ms_exact / steps,
                       "note": "float32 storage, double local arithmetic in the reference's "
                               "operation order (bit-identical to native_relative.cpp)"},
        "fp64_storage_solve": {"ms_per_rk2_step": ms64 / steps64, "steps": steps64},
    }


# pair_value of csrc/semilag5d_tiled.cu: successor position (2 packed FMA
# pairs, 8), floor and weights (3 packed adds and a subtraction, 8), three
# packed bilinear lerps (18) and the heading lerp (3)
SL_FLOPS_PER_EVAL = 37
SL_SMEM_BYTES_PER_EVAL = 4 * 8 + 32


def semilag_cpu_baseline(grid, dt, mode, sample_cells=1 << 17):
    """The FP64 oracle (oracle/semilag5d.c, OpenMP) on a bounded sample: one
    backup of `sample_cells` random cells of the same grid and field."""
    from tests import oracle_lib

    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    o = oracle_lib.load()
    omode = oracle_lib.SL_TUBE if mode == "tube" else oracle_lib.SL_MINTIME
    cfg = o.sl_cfg(a3_config(), grid, dt, omode)
    V = o.sl_init(cfg, grid.states)
    cells = np.random.default_rng(0).choice(grid.states, size=sample_cells, replace=False)
    o.sl_backup_cells(cfg, V, cells[:1024])  # warm-up
    t0 = time.perf_counter()
    o.sl_backup_cells(cfg, V, cells)
    seconds = time.perf_counter() - t0
    return {"value": sample_cells / seconds, "unit": METRIC, "cores": threads,
            "kind": "port",
            "sample": (f"oracle/semilag5d.c (FP64; the reference has no 5D semi-Lagrangian "
                       f"solver): one {mode} backup of {sample_cells} random cells of the "
                       f"{grid.states}-cell grid, {seconds:.3f} s on {threads} threads")}


def semilag_section(with_cpu=True):
    """Relative 5D semi-Lagrangian min-max backups on the 89M-cell grid: the
    tube functional to the 3.0 s horizon at the interpolation-CFL dt
    (ceil(3.0 / dt) backups from the capture field), device time."""
    import math

    import torch
    from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
    from pursuit_evasion_b200.reversible.semilag import SemiLagrangianSolver

    grid = RelativeGrid(**GRID)
    with SemiLagrangianSolver(a3_config(), grid, mode="tube") as s:
        stream = _timing_stream()
        s.set_stream(stream.cuda_stream)
        s.set_skip(False)  # every cell is backed up in every timed backup
        backups = math.ceil(HORIZON / s.dt - 1e-9)
        s.initialize()
        s.iterate(3, tol=0.0, check_every=3)  # warm-up
        s.initialize()
        s.profile(True)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        s.iterate(backups, tol=0.0, check_every=backups)
        t1.record(stream)
        torch.cuda.synchronize()
        ms_total = t0.elapsed_time(t1)
        ms, n = s.kernel_time()
        evaluations = s.evaluations()
        s.profile(False)
        dt, kernel = s.dt, s.kernel
    cells = grid.states
    peak, _ = measured_peaks()
    achieved = 8 * cells * n / (ms / 1e3) / 1e9
    # On-chip rates of the tiled backup from its counted action-pair
    # evaluations: each is SL_FLOPS_PER_EVAL FP32 operations and
    # SL_SMEM_BYTES_PER_EVAL bytes of shared-memory reads (the 4 float2
    # corners and the 32-byte pair entry), against the B200's FP32 and
    # shared-memory peaks at the sampled SM clock.
    seconds = ms / 1e3
    sm_clock_ghz = 1.965
    fp32_peak = 148 * 128 * 2 * sm_clock_ghz * 1e9
    smem_peak = 148 * 128 * sm_clock_ghz * 1e9
    flops = evaluations * SL_FLOPS_PER_EVAL / seconds
    smem = evaluations * SL_SMEM_BYTES_PER_EVAL / seconds
    out = {"workload": f"semilag5d tube RelativeGrid(65,48,21,21,8.0) reversible_free_a3, "
                       f"dt {dt:.6f} s (interpolation CFL), {backups} backups = "
                       f"{HORIZON} s horizon, 9x9 held actions, {kernel} kernel",
           "cells": cells, "value": cells * backups / (ms_total / 1e3), "unit": METRIC,
           "ms_per_backup": ms / n,
           "roofline": {"bound": "on-chip (shared-memory gathers / FP32 issue); HBM "
                                 "fraction reported",
                        "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak,
                        "algorithmic_bytes_per_launch": 8 * cells},
           "on_chip": {"evaluations_per_cell": evaluations / (cells * n) if n else None,
                       "flops_per_evaluation": SL_FLOPS_PER_EVAL,
                       "achieved_tflops": flops / 1e12,
                       "fp32_peak_tflops": fp32_peak / 1e12,
                       "fp32_frac": flops / fp32_peak,
                       "smem_bytes_per_evaluation": SL_SMEM_BYTES_PER_EVAL,
                       "achieved_smem_tbs": smem / 1e12,
                       "smem_peak_tbs": smem_peak / 1e12,
                       "smem_frac": smem / smem_peak,
                       "peaks": "148 SMs x (128 FP32 lanes x 2, 128 B shared memory) per "
                                "clock at 1.965 GHz"}}
    if with_cpu:
        try:
            out["cpu_baseline"] = semilag_cpu_baseline(grid, dt, "tube")
        except Exception as exc:  # the oracle library is built by build()
            out["cpu_baseline"] = {"error": repr(exc)}
    return out


def converge_section(samples, epochs):
    """Time to a converged minimum-time table (sup-norm residual < 1e-5) on
    the 89M-cell grid at the interpolation-CFL dt: cold start vs the learned
    warm start (surrogate trained on the same table, and on a coarse-grid
    table whose solve and training are charged to the warm path)."""
    from pursuit_evasion_b200.learned.warm_start import time_to_converged
    from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
    from pursuit_evasion_b200.reversible.semilag import interpolation_cfl_dt

    grid = RelativeGrid(**GRID)
    dt = interpolation_cfl_dt(a3_config(), grid)
    coarse = RelativeGrid(33, 24, 11, 11, GRID["extent"])
    result, net = time_to_converged(a3_config(), grid, dt=dt, tol=1e-5, samples=samples,
                                    epochs=epochs, batch=8192, coarse_grid=coarse)
    return result, net


def learned_section(net5, samples, epochs, batch=8192, steps8d=200):
    """The learned surrogate beyond the 5D warm start: (1) trained by the
    package's kernels on 2^22 node samples of the 8D contact table
    (WorldGrid(11,9,7,7,3.0) after `steps8d` RK2 steps from the rectangle
    contact field), its error against that table on every node; (2) online
    query latency of the 5D surrogate `net5` for batches of 4096 relative
    states (encode + four tensor-core layers + head), CUDA events per query,
    training charged separately."""
    import torch
    from pursuit_evasion_b200.learned.mlp import ValueMLP
    from pursuit_evasion_b200.learned.train import (
        WorldNodeSampler, predict_nodes, predict_states, train)
    from pursuit_evasion_b200.reversible.world_dp import WorldGrid, WorldSolver

    out = {}
    grid = WorldGrid(11, 9, 7, 7, 3.0)
    dev = torch.device("cuda", 0)
    with WorldSolver(a3_config(), grid, avoid=False, fast=True) as w:
        w.init_contact((0.5, 0.3), (0.5, 0.3))
        for _ in range(steps8d):
            w.step(w.dt_limit)
        table = torch.from_numpy(w.field().reshape(-1)).to(dev)
    net = ValueMLP(WorldNodeSampler.in_features, seed=0, max_batch=batch)
    losses, train_s = train(net, WorldNodeSampler(a3_config(), grid, table), samples=samples,
                            epochs=epochs, batch=batch)
    net.set_batch(1 << 17)
    pred = predict_nodes(net, WorldNodeSampler(a3_config(), grid),
                         torch.empty(grid.states, device=dev), chunk=1 << 17)
    err = (pred - table).abs()
    out["world8d_training"] = {
        "table": f"WorldGrid(11,9,7,7,3.0) contact game after {steps8d} RK2 steps "
                 f"({grid.states} nodes)",
        "samples": samples, "epochs": epochs, "batch": batch, "train_seconds": train_s,
        "final_mse": losses[-1], "max_abs_error": float(err.max()),
        "mean_abs_error": float(err.mean()),
        "p99_abs_error": float(torch.quantile(err[::64], 0.99))}
    del net, pred, table
    if net5 is not None:
        from pursuit_evasion_b200.reversible.free_dp import RelativeGrid

        g5 = RelativeGrid(**GRID)
        net5.set_batch(4096)
        rng = np.random.default_rng(0)
        lo = np.array([-g5.extent, -g5.extent, -np.pi, -1.0, -0.5])
        hi = np.array([g5.extent, g5.extent, np.pi, 2.0, 1.0])
        states = torch.tensor(rng.uniform(lo, hi, size=(4096, 5)), dtype=torch.float32,
                              device=dev)
        stream = torch.cuda.current_stream(dev)
        for _ in range(10):
            predict_states(net5, a3_config(), g5.extent, states)
        times = []
        for _ in range(200):
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            predict_states(net5, a3_config(), g5.extent, states)
            t1.record(stream)
            t1.synchronize()
            times.append(t0.elapsed_time(t1))
        times = np.array(times)
        out["query_latency"] = {
            "batch": 4096, "queries": len(times), "p50_ms": float(np.median(times)),
            "p95_ms": float(np.quantile(times, 0.95)),
            "states_per_s": 4096 / (float(np.median(times)) / 1e3),
            "surrogate": "5D minimum-time surrogate of the converged section"}
    return out


def batch_section(seed=0, count=256):
    """The batched workload: `count` solves drawn from `seed` (positions
    17-49, headings 12-36, speeds 7-15, accelerations 1.5-4, capture radius
    0.3-0.8, horizon 0.5-2 s, box [-4, 4] m), each to its own horizon, in one
    persistent launch with the float32 cell update; tiles from the
    autotuner."""
    import torch
    from pursuit_evasion_b200.batch import BatchSolver, autotune, draw_batch

    solves = draw_batch(seed, count)
    tiles = autotune.tune(solves, local_precision="float32", per_bucket=4, trial_steps=2,
                          repeats=1)
    with BatchSolver(solves, local_precision="float32") as b:
        stream = _timing_stream()
        b.set_stream(stream.cuda_stream)
        autotune.apply(b, tiles)
        b.initialize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        b.run()
        t1.record(stream)
        b.synchronize()
        ms = t0.elapsed_time(t1)
        info = b.launch_info()
        cells = [b.info(i)["cells"] for i in range(len(solves))]
    return {"workload": f"{count} relative 5D solves from seed {seed} (box [-4, 4] m), RK2 "
                        "ENO/LF float32 cell update, each to its own horizon, one cooperative "
                        "launch in a CUDA graph",
            "value": info["cell_stages"] / (ms / 1e3), "unit": METRIC, "ms": ms,
            "launches": 1, "ctas": info["ctas"], "max_steps": info["max_steps"],
            "cells_total": int(sum(cells)), "cell_stages": info["cell_stages"],
            "tiles": tiles}


def synthetic_vehicle_grid(limits, *, half_width, step, headings, speeds, dt=0.05):
    """A compact-game vehicle grid with the reference solve's shapes
    (local_game/reference.py:176-195: 16 headings, 7 speeds) on a synthetic
    lattice: every lattice state is legal, and the successor of each of the 9
    held controls (accel in {-A, 0, A} x curvature in {-K, 0, K}) is a plain
    arc over dt, interpolated with VehicleGrid.stencil.  The reference builds
    its grids with its native geometry engine (legality, braking backups);
    only the shapes and the stencil structure matter for throughput."""
    from pursuit_evasion_b200.local_game.grid_game import VehicleGrid

    n = int(round(2 * half_width / step))
    x = (np.arange(n + 2) - (n + 1) / 2) * step
    axes = (x, x, np.arange(headings) * 2 * np.pi / headings - np.pi,
            np.linspace(limits.speed_min, limits.speed_max, speeds))
    states = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 4)
    controls = np.array([[a, k] for a in (-limits.acceleration, 0, limits.acceleration)
                         for k in (-limits.max_curvature, 0, limits.max_curvature)])
    v = states[:, None, 3]
    v2 = np.clip(v + controls[None, :, 0] * dt, limits.speed_min, limits.speed_max)
    dist = 0.5 * (v + v2) * dt
    turn = controls[None, :, 1] * dist
    mid = states[:, None, 2] + 0.5 * turn
    nxt = np.stack([states[:, None, 0] + dist * np.cos(mid),
                    states[:, None, 1] + dist * np.sin(mid),
                    np.mod(states[:, None, 2] + turn + np.pi, 2 * np.pi) - np.pi, v2], -1)
    grid = VehicleGrid(axes, states, np.arange(len(states), dtype=np.int32), controls,
                       None, None, None, None)
    ids, w, valid, _, mass = grid.stencil(nxt)
    grid.successors = ids.reshape(len(states), len(controls), 16)
    grid.weights = w.reshape(len(states), len(controls), 16)
    grid.allowed = valid.reshape(len(states), len(controls))
    grid.retained_mass = mass.reshape(len(states), len(controls))
    return grid


def compact_section(backups=5, with_cpu=True):
    """The compact eight-state contact game (local_game/grid_game.py, the
    reference's own semi-Lagrangian min-max kernel): pair-packed domain of
    two synthetic 15 x 15 x 16 x 7 vehicle grids (half width 3.25 m, 0.5 m
    position step, a3 limits, dt 0.05 s) within a 2 m exit radius, 0.8 x 0.5
    / 0.4 x 0.25 m footprints; device time of `backups` fused backups."""
    import torch
    from pursuit_evasion_b200.local_game.geometry import CircleArena
    from pursuit_evasion_b200.local_game.grid_game import (
        PairDomain, backup_packed, initialize_packed, packed_gpu_arrays)

    config = a3_config()
    p = synthetic_vehicle_grid(config.pursuer, half_width=3.25, step=0.5, headings=16, speeds=7)
    e = synthetic_vehicle_grid(config.evader, half_width=3.25, step=0.5, headings=16, speeds=7)
    domain = PairDomain.build(p, e, 2.0)
    arena = CircleArena([], 3.25)
    a = packed_gpu_arrays(p, e, domain, max_gb=60)
    stream = _timing_stream()
    a.set_stream(stream.cuda_stream)
    initialize_packed(a, p, e, domain, arena)
    backup_packed(a, p, e, domain)  # warm-up
    a.profile(True)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(backups):
        backup_packed(a, p, e, domain)
    t1.record(stream)
    a.synchronize()
    ms = t0.elapsed_time(t1)
    kms, launches = a.kernel_time()
    a.profile(False)
    pairs = domain.states
    peak, _ = measured_peaks()
    out = {"workload": "compact8d packed contact game, synthetic 15x15x16x7 vehicle grids "
                       "(25,200 states each, 9 held controls, 16-vertex stencils), exit "
                       f"radius 2 m, {backups} backups, float32",
           "pairs": int(pairs), "value": pairs * backups / (ms / 1e3),
           "unit": "pair-backups/s", "ms_per_backup": ms / backups,
           "roofline": {"bound": "L2 gathers / issue; HBM fraction reported",
                        "achieved": 8 * pairs * launches / (kms / 1e3) / 1e9, "peak": peak,
                        "unit": "GB/s",
                        "frac": 8 * pairs * launches / (kms / 1e3) / 1e9 / peak,
                        "algorithmic_bytes_per_launch": 8 * pairs}}
    if with_cpu:
        import importlib.util

        spec = importlib.util.spec_from_file_location(
            "compact_game_oracle", REPO / "oracle" / "compact_game.py")
        cg = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(cg)
        flat = a["current"].get().astype(np.float64)
        pd = {k: np.asarray(getattr(p, k)) for k in ("states", "successors", "weights", "allowed")}
        ed = {k: np.asarray(getattr(e, k)) for k in ("states", "successors", "weights", "allowed")}
        dd = {k: getattr(domain, k) for k in ("p_position", "lookup", "e_indices", "counts",
                                              "offsets")}
        dd["exit_radius"] = domain.exit_radius
        ips = np.random.default_rng(0).choice(len(p.states), size=16, replace=False)
        t = time.perf_counter()
        cg.backup_packed(flat, pd, ed, dd, ips=ips)
        seconds = time.perf_counter() - t
        sample = int(sum(domain.offsets[i + 1] - domain.offsets[i] for i in ips))
        out["cpu_baseline"] = {
            "value": sample / seconds, "unit": "pair-backups/s", "cores": 1, "kind": "port",
            "sample": f"oracle/compact_game.py (NumPy FP64; the reference runs this game "
                      f"only on the GPU): the pairs of 16 random pursuer states "
                      f"({sample} pairs), {seconds:.2f} s"}
    a.close()
    return out


def square6d_section(horizon=2.0, with_cpu=True):
    """The legacy 6D square game on the reference's default grid (17
    positions, 16 headings: 21,381,376 cells), default GameConfig, order 2,
    CFL 0.8, `horizon` seconds: device time of the reference-order stage
    (bit-identical to native_square.cpp), with the reference executable
    itself (oracle/_ref/square6d, all host threads, 0.2 s) beside it."""
    import subprocess
    import tempfile
    from pursuit_evasion_b200.dp.grid import GridSpec
    from pursuit_evasion_b200.dp.native import SquareSolver
    from pursuit_evasion_b200.model import GameConfig

    grid = GridSpec(17, 16, 3.5)
    with SquareSolver(GameConfig(), grid) as s:
        s.initialize()
        s.advance(0.1)  # warm-up
        s.synchronize()
        s.initialize()
        s.profile(True)
        t0 = time.perf_counter()
        s.advance(horizon)
        s.synchronize()
        wall = time.perf_counter() - t0
        kms, launches = s.kernel_time()
        steps = s.steps
        s.profile(False)
    cells = grid.states
    peak, _ = measured_peaks()
    algorithmic = (8 + 12) * cells * steps
    out = {"workload": f"square6d GridSpec(17,16,3.5) default GameConfig, order 2, CFL 0.8, "
                       f"{horizon} s = {steps} RK2 steps, float32 reference order",
           "cells": cells, "value": cells * launches / (kms / 1e3), "unit": METRIC,
           "ms_per_rk2_step": kms / steps, "wall_seconds": wall,
           "roofline": {"bound": "hbm", "achieved": algorithmic / (kms / 1e3) / 1e9,
                        "peak": peak, "unit": "GB/s",
                        "frac": algorithmic / (kms / 1e3) / 1e9 / peak}}
    exe = REPO / "oracle" / "_ref" / "square6d"
    if with_cpu and exe.exists():
        threads = os.cpu_count() or 1
        with tempfile.TemporaryDirectory() as tmp:
            subprocess.run([str(exe), "--horizon", "0.2", "--output-dt", "0.1", "--threads",
                            str(threads), "--history", "0", "--output", tmp + "/o"],
                           check=True, capture_output=True)
            timing = json.loads(Path(tmp + "/o/native_timing.json").read_text())
        value = cells * timing["internal_steps"] * 2 / timing["update_seconds"]
        out["cpu_baseline"] = {
            "value": value, "unit": METRIC, "cores": threads, "kind": "reference",
            "sample": f"native_square.cpp built from the reference sources, same grid, 0.2 s = "
                      f"{timing['internal_steps']} RK2 steps, update loop "
                      f"{timing['update_seconds']:.2f} s on {threads} threads"}
    return out


def run_case(name, repeats):
    """A short, fixed launch sequence of one kernel for profilers (ncu):
    no timing, no JSON line.  One warm-up launch then `repeats` launches of
    the kernel on the full-size workload of that kernel."""
    import torch

    torch.cuda.set_device(0)
    config = a3_config()
    if name == "relative5d":
        from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
        from pursuit_evasion_b200.reversible.relative_solver import RelativeSolver

        with RelativeSolver(config, RelativeGrid(**GRID)) as s:
            s.initialize()
            for _ in range(1 + repeats):  # RK2 steps: two stage launches each
                s.step(s.cfl_dt_limit)
            s.synchronize()
    elif name in ("semilag5d", "semilag5d-generic"):
        from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
        from pursuit_evasion_b200.reversible.semilag import SemiLagrangianSolver

        with SemiLagrangianSolver(config, RelativeGrid(**GRID), mode="tube") as s:
            s.set_kernel("generic" if name.endswith("generic") else "auto")
            s.initialize()
            s.iterate(1 + repeats, tol=0.0, check_every=1 + repeats)
    elif name in ("world8d", "world8d-fast"):
        from pursuit_evasion_b200.reversible.world_dp import WorldGrid, WorldSolver

        with WorldSolver(config, WorldGrid(11, 9, 7, 7, 3.0), avoid=False,
                         fast=name.endswith("fast")) as s:
            s.init_contact((0.5, 0.3), (0.5, 0.3))
            for _ in range(1 + repeats):
                s.step(s.dt_limit)
            s.synchronize()
    elif name == "compact8d":
        from pursuit_evasion_b200.local_game.geometry import CircleArena
        from pursuit_evasion_b200.local_game.grid_game import (
            PairDomain, backup_packed, initialize_packed, packed_gpu_arrays)

        p = synthetic_vehicle_grid(config.pursuer, half_width=3.25, step=0.5, headings=16,
                                   speeds=7)
        e = synthetic_vehicle_grid(config.evader, half_width=3.25, step=0.5, headings=16,
                                   speeds=7)
        domain = PairDomain.build(p, e, 2.0)
        a = packed_gpu_arrays(p, e, domain, max_gb=60)
        initialize_packed(a, p, e, domain, CircleArena([], 3.25))
        for _ in range(1 + repeats):
            backup_packed(a, p, e, domain)
        a.synchronize()
        a.close()
    elif name == "square6d":
        from pursuit_evasion_b200.dp.grid import GridSpec
        from pursuit_evasion_b200.dp.native import SquareSolver
        from pursuit_evasion_b200.model import GameConfig

        with SquareSolver(GameConfig(), GridSpec(17, 16, 3.5)) as s:
            s.initialize()
            for _ in range(1 + repeats):
                s.advance(s.time + s.dt_limit)
            s.synchronize()
    elif name == "mlp":
        from pursuit_evasion_b200.learned.mlp import ValueMLP

        net = ValueMLP(6, seed=0, max_batch=8192)
        net.feat.normal_()
        net.target.normal_()
        for step in range(1, 2 + repeats):
            net.loss.zero_()
            net.forward(8192, target=True)
            net.backward(8192)
            net.set_step(step)
            net.adam(lr=1e-3)
        torch.cuda.synchronize()
    else:
        raise SystemExit(f"unknown case {name}")
    print(f"case {name}: ok", flush=True)


def run_sharded(args, world, rank, local, *, backend="nccl", shard_factory=None, grid=None):
    """`--gpus N` (N > 1, the default mode): ONE config-2 table solved by N
    ranks, each owning a contiguous range of pursuer-speed (vP) slabs with
    `order` halo slabs per neighbour, refreshed after every stage by NCCL
    send/recv between neighbouring ranks; the residual is an all-reduce max
    (pursuit_evasion_b200.reversible.sharded).  Strong scaling: the total
    work is fixed, `value` = all cells x stages / the slowest rank's device
    time.  `e2e` adds, per solve, each rank's upload of its buffer slabs of
    the initial field and the read-back of its owned slabs of the final
    field and arrival times.  The GPU stage kernel is the single-grid one, so
    the table is bit-identical to the one-GPU solve.  The halo slabs are
    copied into each rank's own buffer: every load of the stage kernel reads
    this GPU's memory.  `backend`, `shard_factory` and `grid` let CPU tests
    drive the same code with gloo ranks and oracle shards."""
    import datetime

    import torch
    import torch.distributed as dist

    from pursuit_evasion_b200.reversible.free_dp import RelativeGrid, output_times
    from pursuit_evasion_b200.reversible.sharded import (
        DistExchange, RelativeShard, ShardedSolver, partition)

    gpu = backend == "nccl"
    if gpu:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local))
    elif not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    grid = grid or RelativeGrid(**GRID)
    ranges = partition(grid.p_speeds, world, 2)
    begin, end = ranges[rank]
    if shard_factory is None:
        def shard_factory(b, e):
            return RelativeShard(a3_config(), grid, b, e, local_precision=args.precision,
                                 device=local)
    shard = shard_factory(begin, end)
    frame_times = output_times(HORIZON, OUTPUT_DT)[1:]
    cells = grid.states
    try:
        solver = ShardedSolver([shard], DistExchange(shard))
        stream = solver._stream  # the shard's stages and the NCCL exchanges

        def one_solve(initial=None, read_back=False):
            shard.initialize(initial)
            solver.time, solver.steps = 0.0, 0
            for goal in frame_times:
                solver.advance(goal)
            if read_back:
                shard.field()
                shard.arrival()

        def timed(count, **kw):
            """Device time of `count` solves on the solver's stream (CUDA
            events), or wall time on CPU ranks."""
            if gpu:
                torch.cuda.synchronize()
            dist.barrier()
            if gpu:
                t0, t1 = (torch.cuda.Event(enable_timing=True),
                          torch.cuda.Event(enable_timing=True))
                t0.record(stream)
            else:
                w0 = time.perf_counter()
            for _ in range(count):
                one_solve(**kw)
            if gpu:
                t1.record(stream)
                torch.cuda.synchronize()
                return t0.elapsed_time(t1)
            return (time.perf_counter() - w0) * 1e3

        for _ in range(args.warmup):
            one_solve()
        steps = solver.steps
        clocks = ClockSampler(local) if gpu else None
        if clocks:
            clocks.start()
        ms = timed(args.steps)
        clock_info = clocks.stop() if clocks else None
        e2e_ms = timed(args.steps, initial=shard_initial_field(grid), read_back=True)
        t = torch.tensor([ms, e2e_ms], dtype=torch.float64,
                         device=f"cuda:{local}" if gpu else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms = t.tolist()
        line = None
        if rank == 0:
            backups = cells * 2 * steps * args.steps
            slab = cells // grid.p_speeds
            own = [(e - b) * slab for b, e in ranges]
            buf = [(min(grid.p_speeds, e + 2) - max(0, b - 2)) * slab for b, e in ranges]
            line = {
                "metric": METRIC, "value": backups / (ms / 1e3), "unit": METRIC,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None,
                "dtype": "f32" if args.precision == "float32" else "f32 storage, f64 local",
                "data": "synthetic (deterministic grid, no dataset)",
                "config": bench_config(cells),
                "run": {"stages_per_step": 2 * steps, "precision": args.precision,
                        "parallelism": f"vP slabs x{world} (NCCL halo exchange)",
                        "vp_ranges": [list(r) for r in ranges]},
                "e2e": {"value": backups / (e2e_ms / 1e3), "unit": METRIC,
                        "h2d_bytes_per_step": 4 * sum(buf),
                        "d2h_bytes_per_step": 8 * sum(own),
                        "ms_per_step": e2e_ms / args.steps},
                "gpu_launches": int(world * 2 * steps * args.steps) if gpu else 0,
                "clocks": clock_info,
                "timing": "CUDA events on each rank's solve stream, max over ranks",
            }
            print(json.dumps(line), flush=True)
        dist.barrier()
        return line
    finally:
        if hasattr(shard, "close"):
            shard.close()
        if gpu:
            dist.destroy_process_group()


def shard_initial_field(grid):
    """The capture field hypot(x, y) - r as a host array (the e2e input)."""
    x = np.linspace(-grid.extent, grid.extent, grid.positions)
    plane = (np.hypot(x[None, :], x[:, None]) - A3_LIMITS["capture_radius"]).astype(np.float32)
    reps = grid.states // plane.size
    return np.broadcast_to(plane, (reps,) + plane.shape).reshape(-1)


def run_ours(args, world, rank, local):
    import torch

    from pursuit_evasion_b200 import _native
    from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
    from pursuit_evasion_b200.reversible.relative_solver import RelativeSolver

    torch.cuda.set_device(local)
    # A stream of our own: the solver handles run on it and the timing
    # events are recorded on it (the legacy default stream would neither).
    torch.cuda.set_stream(torch.cuda.Stream(device=local))
    if world > 1:
        import datetime
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    config = a3_config()
    grid = RelativeGrid(**GRID)
    cells = grid.states
    solver = RelativeSolver(config, grid, local_precision=args.precision,
                            device=local)
    stream = _timing_stream()
    solver.set_stream(stream.cuda_stream)
    stages_per_solve = None

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    from pursuit_evasion_b200.reversible.free_dp import output_times

    frame_times = output_times(HORIZON, OUTPUT_DT)[1:]

    def advance_all():
        taken = 0
        for goal in frame_times:
            taken += solver.advance(goal)
        return taken

    def one_solve():
        solver.initialize()
        return advance_all()

    for _ in range(args.warmup):
        steps = one_solve()
    stages_per_solve = 2 * steps
    solver.synchronize()

    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    launches0 = _native.launch_count()
    solver.profile(True)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        one_solve()
    end.record(stream)
    barrier()
    clock_info = clocks.stop()
    launches = _native.launch_count() - launches0
    elapsed_ms = start.elapsed_time(end)
    stage_ms = [solver.kernel_time(0), solver.kernel_time(1)]
    solver.profile(False)
    solver.synchronize()

    # e2e: public API with host buffers, pinned memory both ways.
    host_init = torch.empty(cells, dtype=torch.float32, pin_memory=True)
    host_field = torch.empty(cells, dtype=torch.float32, pin_memory=True)
    host_arrival = torch.empty(cells, dtype=torch.float32, pin_memory=True)
    solver.initialize()
    solver.copy_field_to(host_init.data_ptr())  # the capture field as the input
    init_np = host_init.numpy()
    barrier()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(args.steps):
        solver.initialize(init_np)
        advance_all()
        solver.copy_field_to(host_field.data_ptr())
        solver._lib.pe_relative_copy_arrival(solver._h, host_arrival.data_ptr())
    e_end.record(stream)
    barrier()
    e2e_ms = e_start.elapsed_time(e_end)

    # max over ranks
    elapsed_ms, e2e_ms = max_over_ranks([elapsed_ms, e2e_ms], world)
    backups = cells * stages_per_solve * args.steps * world
    value = backups / (elapsed_ms / 1e3)
    e2e_value = backups / (e2e_ms / 1e3)

    line = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        (ms1, n1), (ms2, n2) = stage_ms
        bytes1, bytes2 = 8 * cells, 12 * cells
        achieved = (bytes1 * n1 + bytes2 * n2) / ((ms1 + ms2) / 1e3) / 1e9
        traffic = profile_traffic()
        roofline = {
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
            "kernel": "rel5_stage_fast_kernel (stage 1 + stage 2)",
            "algorithmic_bytes_per_launch": {"stage1": bytes1, "stage2": bytes2},
            "avg_launch_ms": {"stage1": ms1 / max(n1, 1), "stage2": ms2 / max(n2, 1)},
            "traffic": None if traffic is None else traffic.get("bytes_per_launch"),
        }
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "float32" else "f32 storage, f64 local",
            "data": "synthetic (deterministic grid, no dataset)",
            "config": bench_config(cells),
            "run": {"stages_per_step": stages_per_solve, "precision": args.precision,
                    "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": roofline,
            "e2e": {"value": e2e_value, "unit": METRIC,
                    "h2d_bytes_per_step": 4 * cells,
                    "d2h_bytes_per_step": 8 * cells,
                    "ms_per_step": e2e_ms / args.steps},
            "gpu_launches": int(launches),
            "clocks": clock_info,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        # side measurements are single-GPU; with replicas they would keep the
        # other ranks waiting at the final barrier
        if not args.no_sections and world == 1:
            final_table = host_field.numpy().copy()
            for key, fn in (("fp64_error", lambda: fp64_section(final_table)),
                            ("world8d", world8d_section),
                            ("semilag5d", lambda: semilag_section(not args.no_cpu_baseline)),
                            ("batch", batch_section),
                            ("compact8d", lambda: compact_section(
                                with_cpu=not args.no_cpu_baseline)),
                            ("square6d", lambda: square6d_section(
                                with_cpu=not args.no_cpu_baseline))):
                try:
                    line[key] = fn()
                except Exception as exc:  # report, keep the headline line
                    line[key] = {"error": repr(exc)}
            net5 = None
            if args.converge:
                try:
                    line["converged"], net5 = converge_section(args.samples, args.epochs)
                except Exception as exc:
                    line["converged"] = {"error": repr(exc)}
                try:
                    line["learned"] = learned_section(net5, args.samples, args.epochs)
                except Exception as exc:
                    line["learned"] = {"error": repr(exc)}
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return line


def main():
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--mode", choices=["sharded", "replicas"], default="sharded",
                        help="with --gpus N > 1: one table in vP slabs over the N ranks "
                             "(strong scaling, default) or N independent tables")
    parser.add_argument("--precision", choices=["float32", "float64"],
                        default="float32")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-sections", action="store_true",
                        help="skip the 8D and semi-Lagrangian side measurements")
    parser.add_argument("--converge", action=argparse.BooleanOptionalAction, default=True,
                        help="time-to-converged table, plain vs learned warm start")
    parser.add_argument("--samples", type=int, default=1 << 22)
    parser.add_argument("--epochs", type=int, default=20)
    parser.add_argument("--case", choices=["relative5d", "semilag5d", "semilag5d-generic",
                                           "world8d", "world8d-fast", "mlp", "compact8d",
                                           "square6d"],
                        help="run a short launch sequence of one kernel for a profiler")
    parser.add_argument("--repeats", type=int, default=2)
    args = parser.parse_args()
    if args.case:
        run_case(args.case, args.repeats)
        return
    # At least three warm-up solves are always run.
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
    elif world > 1 and args.mode == "sharded":
        run_sharded(args, world, rank, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
