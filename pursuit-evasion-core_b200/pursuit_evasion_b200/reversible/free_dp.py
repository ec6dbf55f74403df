"""Drop-in `reversible.free_dp` for B200: the relative 5D capture-tube solve.

Same Python API and the same completed-table directory as pursuit-evasion-core
src/pursuit_evasion/reversible/free_dp.py:
    solve(config, grid, output, *, horizon, output_dt, order, cfl, threads,
          history, max_working_gb, disk_reserve_gb) -> meta dict
writing meta.json (schema "reversible_relative5d_v1"), fields.f32
([T, vP, vE, psi, y, x] float32, frame 0 = initial field), final.f32,
arrival.f32, timing.json, progress.jsonl and solver.log, which the reference's
RelativeTable (relative_table.py:11-61) reads.  The reference runs a g++/OpenMP
executable per solve (free_dp.py:259-261); here the per-cell work runs in
hand-written sm_100a kernels behind libpe_b200.so.

Extra keywords (defaults keep the reference behaviour):
    local_precision  "float64" (default) reproduces the reference executable
                     bit for bit; "float32" is the fast path.
    device           CUDA device ordinal.
    tol              stop early once a step changes no cell by tol or more
                     (sup-norm convergence); the last frame is the converged
                     field and meta records `converged_time`.
    warm_start       optional initial field (cells float32) replacing the
                     circular capture field.
    save_final       write final.f32 / arrival.f32 (default True).
"""

from __future__ import annotations

from dataclasses import asdict, dataclass
import hashlib
import json
import math
import os
from pathlib import Path
import queue
import shutil
import threading
import time

import numpy as np

from .model import config_dict
from .relative_solver import PinnedBuffer, RelativeSolver

SCHEMA = "reversible_relative5d_v1"
SOURCE_DIR = Path(__file__).resolve().parents[2] / "csrc"


@dataclass(frozen=True)
class RelativeGrid:
    """Relative grid [vP, vE, psi, y, x]; same fields and checks as
    free_dp.py:23-72 (positions >= 3, headings >= 4, speeds >= 3)."""

    positions: int = 41
    headings: int = 24
    p_speeds: int = 7
    e_speeds: int = 7
    extent: float = 4.0

    def __post_init__(self):
        minimum = {"positions": 3, "headings": 4, "p_speeds": 3, "e_speeds": 3}
        for name, low in minimum.items():
            value = getattr(self, name)
            if isinstance(value, bool) or int(value) != value or value < low:
                raise ValueError(f"Invalid {name}: {value}")
        if not np.isfinite(self.extent) or self.extent <= 0:
            raise ValueError("extent must be finite and positive")

    @property
    def shape(self):
        return (self.p_speeds, self.e_speeds, self.headings, self.positions,
                self.positions)

    @property
    def states(self):
        return math.prod(self.shape)

    def axes(self, config):
        p, e = config.pursuer, config.evader
        return (
            np.linspace(p.speed_min, p.speed_max, self.p_speeds),
            np.linspace(e.speed_min, e.speed_max, self.e_speeds),
            np.linspace(-np.pi, np.pi, self.headings, endpoint=False),
            np.linspace(-self.extent, self.extent, self.positions),
            np.linspace(-self.extent, self.extent, self.positions),
        )

    def to_dict(self):
        return asdict(self)


def output_times(horizon, output_dt):
    """Frame times min(k * output_dt, horizon), k = 0..ceil(h/dt - 1e-10)."""
    count = math.ceil(horizon / output_dt - 1e-10)
    return np.minimum(np.arange(count + 1) * output_dt, horizon)


def physics_signature(config):
    """Table-compatibility signature (same keys as free_dp.py:80-96)."""
    signature = {"capture_radius": float(config.capture_radius)}
    for role in ("pursuer", "evader"):
        limits = getattr(config, role)
        signature[role] = {
            k: float(getattr(limits, k))
            for k in ("speed_min", "speed_max", "acceleration", "max_curvature")
        }
    if config.capture_rule != "center_distance":
        signature["capture_rule"] = config.capture_rule
    return signature


def _validate(config, grid, horizon, output_dt, order, cfl, threads):
    """Option checks of free_dp.py:99-128 (ValueError on any failure)."""
    numbers = [horizon, output_dt, cfl, config.capture_radius, grid.extent]
    for limits in (config.pursuer, config.evader):
        numbers += [limits.speed_min, limits.speed_max, limits.acceleration,
                    limits.max_curvature]
        if (limits.speed_min >= limits.speed_max or limits.acceleration <= 0
                or limits.max_curvature <= 0):
            raise ValueError("Invalid vehicle limits")
    if (not np.isfinite(numbers).all() or horizon <= 0 or output_dt <= 0
            or not 0 < cfl <= 1):
        raise ValueError("Invalid numeric solve options")
    if (not 0 < config.capture_radius < grid.extent or order not in (1, 2)
            or threads < 1):
        raise ValueError("Invalid radius, order or thread count")


def _source_digest():
    digest = hashlib.sha256()
    for path in sorted(SOURCE_DIR.glob("relative5d*")) + sorted(
            SOURCE_DIR.glob("capi_relative.cu")):
        digest.update(path.read_bytes())
    return digest.hexdigest()


def solve(
    config,
    grid,
    output,
    *,
    horizon=2.0,
    output_dt=0.1,
    order=2,
    cfl=0.8,
    threads=4,
    history=True,
    max_working_gb=8.0,
    disk_reserve_gb=10.0,
    local_precision="float64",
    device=0,
    tol=None,
    warm_start=None,
    save_final=True,
    probes=None,
    capture_footprints=None,
    exit_radius=None,
    scheme="eno_lf",
):
    """Compute a new relative table directory on the GPU.

    Refuses an existing non-empty output (FileExistsError), a working set
    above max_working_gb (MemoryError, before anything is created) and too
    little disk (OSError), like free_dp.py:145-176.  `threads` is accepted
    for signature compatibility and recorded; the GPU does not use it.

    The reference's GPU solve (gpu_relative.py:67-101) adds three keywords,
    accepted here with its meaning and errors: `capture_footprints` =
    (pursuer, evader) Footprints for a "rectangle_contact" configuration
    (the capture field becomes the oriented-rectangle separation over every
    heading); `exit_radius` = R in (0, extent): cells with x^2 + y^2 > R^2
    start at and stay at R; `probes` = relative states [n, 5] (x, y, psi,
    vP, vE) whose multilinear values are written to probes.f64 after every
    frame.  `warm_start`, when given, replaces the initial field; the exit
    still holds in every stage.

    scheme="semi_lagrangian" fills the same table with the semi-Lagrangian
    min-max backup (the tube form, V' = min(V, min_u max_w V(successor))):
    each output interval is split into equal held-command steps no longer
    than the interpolation CFL step, arrival times follow the same crossing
    rule, and two extra files hold the optimal pursuer / evader actions of
    the last backup (policy_p.u8, policy_e.u8: catalogue index
    3 * acceleration + curvature, each in (-, 0, +) order) and residuals.f64
    the sup-norm change of each frame's last backup.  It takes no `tol` and
    no `exit_radius`.
    """
    solve_started = time.perf_counter()
    if config.capture_rule == "rectangle_contact" and capture_footprints is None:
        raise ValueError("Rectangle capture requires explicit P/E footprints")
    if config.capture_rule == "center_distance" and capture_footprints is not None:
        raise ValueError("Declare rectangle_contact in the configuration")
    if config.capture_rule not in ("center_distance", "rectangle_contact"):
        raise ValueError("Unknown capture rule")
    if exit_radius is not None and not 0 < exit_radius < grid.extent:
        raise ValueError("Local exit radius must lie inside the numerical grid")
    if scheme not in ("eno_lf", "semi_lagrangian"):
        raise ValueError("scheme must be 'eno_lf' or 'semi_lagrangian'")
    if scheme == "semi_lagrangian" and (tol is not None or exit_radius is not None):
        raise ValueError("tol and exit_radius apply to scheme='eno_lf' only")
    _validate(config, grid, horizon, output_dt, order, cfl, threads)
    if (not np.isfinite([max_working_gb, disk_reserve_gb]).all()
            or max_working_gb <= 0 or disk_reserve_gb < 0):
        raise ValueError("Invalid memory/disk guards")
    if tol is not None and not (np.isfinite(tol) and tol > 0):
        raise ValueError("tol must be a positive finite number")
    if local_precision not in ("float32", "float64"):
        raise ValueError("local_precision must be float32 or float64")
    output = Path(output).resolve()
    if output.exists() and any(output.iterdir()):
        raise FileExistsError(f"Preserve existing output: {output}")
    times = output_times(horizon, output_dt)
    N = grid.states
    working = N * (15 if scheme == "semi_lagrangian" else 12)
    probe_states = probe_indices = probe_weights = None
    if probes is not None:
        probe_states, probe_indices, probe_weights = probe_stencils(config, grid, probes)
    storage = N * 4 * ((2 if save_final else 0) + (len(times) if history else 0)) + (
        0 if probe_states is None else 8 * len(probe_states) * len(times)) + (
        2 * N if scheme == "semi_lagrangian" else 0)
    if working > max_working_gb * 1e9:
        raise MemoryError(
            f"Core arrays need {working / 1e9:.3f} GB, above guard {max_working_gb}"
        )
    output.parent.mkdir(parents=True, exist_ok=True)
    free = shutil.disk_usage(output.parent).free
    if storage + disk_reserve_gb * 1e9 > free:
        raise OSError(
            f"Output needs {storage / 1e9:.3f} GB while retaining "
            f"{disk_reserve_gb} GB disk reserve"
        )
    initial = None
    if warm_start is not None:
        initial = np.ascontiguousarray(warm_start, dtype=np.float32).reshape(-1)
        if initial.size != N or not np.isfinite(initial).all():
            raise ValueError("warm_start must be a finite field of grid.states cells")

    if scheme == "semi_lagrangian":
        return _solve_semilag(config, grid, output, times, initial, history=history,
                              save_final=save_final, capture_footprints=capture_footprints,
                              probe_states=probe_states,
                              probe=None if probe_states is None else
                              (probe_indices, probe_weights),
                              device=device, working=working, storage=storage,
                              solve_started=solve_started, horizon=horizon,
                              output_dt=output_dt)
    alloc_started = time.perf_counter()
    solver = RelativeSolver(config, grid, order=order, cfl=cfl,
                            local_precision=local_precision, device=device)
    output.mkdir(exist_ok=True)
    meta = {"schema": SCHEMA, "status": "running"}
    try:
        solver.set_exit(exit_radius)
        if initial is not None:
            solver.initialize(initial)
        else:
            solver.initialize_plane(capture_plane(config, grid, capture_footprints, exit_radius))
        allocation_seconds = time.perf_counter() - alloc_started
        meta.update({
            "schema": SCHEMA,
            "backend": "b200_cuda",
            "local_precision": local_precision,
            "config": config_dict(config),
            "physics": physics_signature(config),
            "grid": grid.to_dict(),
            "shape": list(grid.shape),
            "state_order": ["x", "y", "psi", "vP", "vE"],
            "axis_order": ["vP", "vE", "psi", "y", "x"],
            "axes": [a.tolist() for a in grid.axes(config)],
            "horizon": horizon,
            "output_dt": output_dt,
            "times": times.tolist(),
            "order": order,
            "cfl": cfl,
            "threads": threads,
            "history_saved": bool(history),
            "dtype": "float32",
            "target": "physical_capture_only",
            "scheme": "eno_lf",
            "capture_rule": config.capture_rule,
            "capture_footprints": None if capture_footprints is None else {
                "pursuer": capture_footprints[0].to_dict(),
                "evader": capture_footprints[1].to_dict()},
            "local_exit_radius": exit_radius,
            "avoid": None,
            "tube_projection": "min over every internal update",
            "position_boundary":
                "one-sided linear extrapolation; outside queries unresolved",
            "speed_boundary":
                "acceleration restricted to inward or zero at speed limits",
            "heading_boundary": "periodic",
            "source_sha256": _source_digest(),
            "source_file": None,
            "compile_seconds": 0.0,
            "warm_start": warm_start is not None,
            "tol": tol,
            "cfl_dt_limit": solver.cfl_dt_limit,
            "predicted_working_bytes": working,
            "predicted_output_bytes": storage,
            "device": int(device),
            "status": "running",
            "probe_states": None if probe_states is None else probe_states.tolist(),
        })
        (output / "meta.json").write_text(json.dumps(meta, indent=2) + "\n")
        probe = None if probe_states is None else (probe_indices, probe_weights)
        meta.update(_run(solver, output, times, history=history, tol=tol,
                         save_final=save_final, probe=probe))
        meta["allocation_seconds"] = allocation_seconds
        meta["status"] = "complete"
        if meta["frames"] != len(meta["times"]):
            meta["status"] = "failed"
            meta["failure"] = "Output time count mismatch"
    except Exception as exc:
        meta.update(status="failed", failure=str(exc))
        (output / "meta.json").write_text(json.dumps(meta, indent=2) + "\n")
        raise RuntimeError(f"Relative solve failed: {exc}") from exc
    finally:
        solver.close()
    meta["total_wall_seconds"] = time.perf_counter() - solve_started
    (output / "meta.json").write_text(json.dumps(meta, indent=2) + "\n")
    if meta["status"] != "complete":
        raise RuntimeError(f"Relative solve failed: {output / 'solver.log'}")
    return meta


class _HistoryWriter:
    """Writes the output frames of fields.f32 while the solver runs on: each
    frame is snapshotted on the device (two slots), copied to page-locked
    host memory on a separate stream and written by this thread, in order.
    The reference stops its solver for every history write
    (native_relative.cpp:111-120)."""

    def __init__(self, solver, file, count):
        self.solver, self.file = solver, file
        self.buffers = [PinnedBuffer(count), PinnedBuffer(count)]
        self.free = threading.Semaphore(2)
        self.queue = queue.Queue()
        self.next_slot = 0
        self.transfer_seconds = self.write_seconds = 0.0
        self.error = None
        self.thread = threading.Thread(target=self._loop, name="history-writer", daemon=True)
        self.thread.start()

    def submit(self):
        """Queue the solver's current field as the next frame."""
        self.free.acquire()  # a slot whose previous frame has been written
        if self.error is not None:
            self.free.release()
            raise self.error
        slot, self.next_slot = self.next_slot, self.next_slot ^ 1
        self.solver.snapshot(slot)
        self.queue.put(slot)

    def _loop(self):
        while True:
            slot = self.queue.get()
            if slot is None:
                return
            try:
                if self.error is None:
                    t0 = time.perf_counter()
                    self.solver.copy_snapshot(slot, self.buffers[slot].ptr)
                    t1 = time.perf_counter()
                    self.buffers[slot].array.tofile(self.file)
                    self.transfer_seconds += t1 - t0
                    self.write_seconds += time.perf_counter() - t1
            except BaseException as exc:  # reported by submit / close
                self.error = exc
            finally:
                self.free.release()

    def close(self):
        self.queue.put(None)
        self.thread.join()
        for b in self.buffers:
            b.close()
        if self.error is not None:
            raise self.error


def _solve_semilag(config, grid, output, times, initial, *, history, save_final,
                   capture_footprints, probe_states, probe, device, working, storage,
                   solve_started, horizon, output_dt):
    """The table of free_dp.solve from the semi-Lagrangian tube backup."""
    from .semilag import SemiLagrangianSolver, interpolation_cfl_dt

    limit = interpolation_cfl_dt(config, grid)
    N = grid.states
    warm = initial is not None
    if initial is None:
        plane = capture_plane(config, grid, capture_footprints)
        initial = np.ascontiguousarray(np.broadcast_to(plane, grid.shape)).reshape(-1)
    output.mkdir(exist_ok=True)
    meta = {"schema": SCHEMA, "status": "running"}
    solver = None
    files = []
    try:
        alloc_started = time.perf_counter()

        def make(length):
            steps = max(1, int(math.ceil(length / limit - 1e-9)))
            return SemiLagrangianSolver(config, grid, dt=length / steps, mode="tube",
                                        device=device), steps

        solver, per_frame = make(output_dt)
        segment = output_dt
        solver.initialize(initial)
        solver.track_arrival(start_time=0.0)
        allocation_seconds = time.perf_counter() - alloc_started
        meta.update({
            "schema": SCHEMA,
            "backend": "b200_cuda",
            "scheme": "semi_lagrangian",
            "local_precision": "float32",
            "config": config_dict(config),
            "physics": physics_signature(config),
            "grid": grid.to_dict(),
            "shape": list(grid.shape),
            "state_order": ["x", "y", "psi", "vP", "vE"],
            "axis_order": ["vP", "vE", "psi", "y", "x"],
            "axes": [a.tolist() for a in grid.axes(config)],
            "horizon": horizon,
            "output_dt": output_dt,
            "times": times.tolist(),
            "history_saved": bool(history),
            "dtype": "float32",
            "target": "physical_capture_only",
            "capture_rule": config.capture_rule,
            "capture_footprints": None if capture_footprints is None else {
                "pursuer": capture_footprints[0].to_dict(),
                "evader": capture_footprints[1].to_dict()},
            "local_exit_radius": None,
            "avoid": None,
            "tube_projection": "min over every internal update",
            "position_boundary": "successors interpolated inside the grid, clamped at its edges",
            "speed_boundary": "speed saturates at its limits along the held command",
            "heading_boundary": "periodic",
            "interpolation_cfl_dt": limit,
            "policy_files": ["policy_p.u8", "policy_e.u8"],
            "policy_catalogue": "3 * i_acceleration + i_curvature, each index over (-, 0, +)",
            "source_sha256": _source_digest(),
            "warm_start": warm,
            "predicted_working_bytes": working,
            "predicted_output_bytes": storage,
            "device": int(device),
            "status": "running",
            "probe_states": None if probe_states is None else probe_states.tolist(),
        })
        (output / "meta.json").write_text(json.dumps(meta, indent=2) + "\n")
        host = np.empty(N, np.float32)
        history_file = (output / "fields.f32").open("wb") if history else None
        probe_file = (output / "probes.f64").open("wb") if probe is not None else None
        files = [f for f in (history_file, probe_file) if f is not None]
        residuals = []
        update_seconds = transfer_seconds = write_seconds = 0.0
        started = time.perf_counter()

        def save_frame():
            nonlocal transfer_seconds, write_seconds
            if history_file is None and probe_file is None:
                return
            t0 = time.perf_counter()
            solver.value(host)
            t1 = time.perf_counter()
            transfer_seconds += t1 - t0
            if history_file is not None:
                host.tofile(history_file)
            if probe_file is not None:
                (host[probe[0]].astype(np.float64) * probe[1]).sum(1).tofile(probe_file)
                probe_file.flush()
            write_seconds += time.perf_counter() - t1

        save_frame()
        steps = 0
        with (output / "progress.jsonl").open("w") as progress:
            for index, goal in enumerate(times[1:], start=1):
                length = float(goal - times[index - 1])
                if abs(length - segment) > 1e-9 * max(1.0, segment):
                    # a shorter last interval: continue on a solver with its step
                    nxt, per_frame = make(length)
                    nxt.initialize_device(solver.device_value_ptr())
                    nxt.track_arrival(solver.arrival(), start_time=float(times[index - 1]))
                    solver.close()
                    solver, segment = nxt, length
                t0 = time.perf_counter()
                last = index == len(times) - 1
                for k in range(per_frame):
                    solver.backup(with_policy=last and k == per_frame - 1)
                residuals.append(solver.residual())
                update_seconds += time.perf_counter() - t0
                steps += per_frame
                save_frame()
                if index % 5 == 0 or last:
                    resolved = int(np.isfinite(solver.arrival()).sum())
                    progress.write(json.dumps(dict(
                        time=float(goal), steps=steps, resolved=resolved,
                        elapsed_seconds=time.perf_counter() - started)) + "\n")
                    progress.flush()
        for f in files:
            f.close()
        files = []
        (output / "solver.log").write_text(
            f"semi_lagrangian steps={steps} frames={len(times)}\n")
        np.asarray(residuals, np.float64).tofile(output / "residuals.f64")
        t0 = time.perf_counter()
        if save_final:
            solver.value(host).tofile(output / "final.f32")
            solver.arrival(host).tofile(output / "arrival.f32")
        if len(times) > 1:
            pol_p, pol_e = solver.policy()
            np.ascontiguousarray(pol_p, np.uint8).tofile(output / "policy_p.u8")
            np.ascontiguousarray(pol_e, np.uint8).tofile(output / "policy_e.u8")
        final_write = time.perf_counter() - t0
        timing = {
            "states": N,
            "working_array_bytes": working,
            "step_dt": solver.dt,
            "internal_steps": steps,
            "frames": len(times),
            "update_seconds": update_seconds,
            "device_to_host_seconds": transfer_seconds,
            "history_write_seconds": write_seconds,
            "final_write_seconds": final_write,
            "elapsed_seconds": time.perf_counter() - started,
            "last_step_residual": residuals[-1] if residuals else 0.0,
            "cell_backups_per_second": N * steps / max(update_seconds, 1e-12),
        }
        (output / "timing.json").write_text(json.dumps(timing) + "\n")
        meta.update(timing)
        meta["allocation_seconds"] = allocation_seconds
        meta["status"] = "complete"
    except Exception as exc:
        meta.update(status="failed", failure=str(exc))
        (output / "meta.json").write_text(json.dumps(meta, indent=2) + "\n")
        raise RuntimeError(f"Relative solve failed: {exc}") from exc
    finally:
        for f in files:
            f.close()
        if solver is not None:
            solver.close()
    meta["total_wall_seconds"] = time.perf_counter() - solve_started
    (output / "meta.json").write_text(json.dumps(meta, indent=2) + "\n")
    return meta


def capture_plane(config, grid, capture_footprints=None, exit_radius=None):
    """The initial (y, x) plane, or (psi, y, x) block for rectangle contact,
    as the reference GPU solve builds it (gpu_relative.py:165-175): centre
    distance minus the capture radius, or the oriented-rectangle separation
    of an evader at (x, y, psi) from a pursuer at the origin; beyond the
    local exit the value is the exit radius."""
    n = grid.positions
    dx = 2 * grid.extent / (n - 1)
    coord = -grid.extent + np.arange(n) * dx
    plane = (np.hypot(coord[:, None], coord[None, :]) - config.capture_radius).astype(np.float32)
    xx, yy = np.meshgrid(coord, coord)
    if capture_footprints is not None:
        from ..local_game.geometry import rectangle_separation

        psi = grid.axes(config)[2]
        other = np.zeros((grid.headings, n, n, 4))
        other[..., 0], other[..., 1], other[..., 2] = xx, yy, psi[:, None, None]
        plane = rectangle_separation(np.zeros(4), other, *capture_footprints).astype(np.float32)
    if exit_radius is not None:
        plane = np.where(xx * xx + yy * yy > exit_radius ** 2, exit_radius,
                         plane).astype(np.float32)
    return plane


def probe_stencils(config, grid, probes):
    """Validated probe states and their 32-corner multilinear stencils over
    the dense storage order (gpu_relative.py:178-214): positions and speeds
    clamp the cell to the last interval, headings wrap.  Returns (states,
    indices [n, 32] int64, weights [n, 32] float64)."""
    states = np.asarray(probes, dtype=float)
    if (states.ndim != 2 or states.shape[1] != 5 or len(states) > 100000
            or not np.isfinite(states).all()):
        raise ValueError("Probes must be finite relative states[n,5]")
    shape = tuple(grid.shape)
    axes = grid.axes(config)
    corner = (np.arange(32)[:, None] >> np.arange(4, -1, -1)[None, :]) & 1  # [32, 5]
    stride = np.ones(5, np.int64)
    for k in range(3, -1, -1):
        stride[k] = stride[k + 1] * shape[k + 1]
    indices = np.zeros((len(states), 32), np.int64)
    weights = np.ones((len(states), 32))
    storage = states[:, [3, 4, 2, 1, 0]]  # (vP, vE, psi, y, x)
    for k in range(5):
        axis, n = np.asarray(axes[k], dtype=float), shape[k]
        step = axis[1] - axis[0]
        q = storage[:, k]
        if k == 2:
            f = np.mod(q + np.pi, 2 * np.pi) / step
            cell = np.floor(f).astype(np.int64) % n
            frac = f - np.floor(f)
        else:
            if np.any((q < axis[0]) | (q > axis[-1])):
                raise ValueError("A probe lies outside the grid")
            f = (q - axis[0]) / step
            cell = np.minimum(np.floor(f).astype(np.int64), n - 2)
            frac = f - cell
        node = cell[:, None] + corner[None, :, k]
        if k == 2:
            node %= n
        indices += node * stride[k]
        weights *= np.where(corner[None, :, k] == 1, frac[:, None], 1 - frac[:, None])
    return states, indices, weights


def _run(solver, output, times, *, history, tol, save_final, probe=None):
    """Frame loop: advance to each output time, save the frame, log progress."""
    N = solver.cells
    host = np.empty(N, np.float32)
    write_seconds = update_seconds = transfer_seconds = 0.0
    probe_seconds = 0.0
    probe_file = (output / "probes.f64").open("wb") if probe is not None else None

    def save_probes():
        nonlocal probe_seconds
        if probe_file is not None:
            t0 = time.perf_counter()
            solver.probe(*probe).tofile(probe_file)
            probe_file.flush()
            probe_seconds += time.perf_counter() - t0

    frames = 1
    converged_time = None
    kept_times = [float(times[0])]
    history_file = (output / "fields.f32").open("wb") if history else None
    writer = None
    log = (output / "solver.log").open("w")
    progress = (output / "progress.jsonl").open("w")
    started = time.perf_counter()
    try:
        save_probes()
        if history_file:
            writer = _HistoryWriter(solver, history_file, N)
            writer.submit()  # frame 0: the initial field
        for index, goal in enumerate(times[1:], start=1):
            t0 = time.perf_counter()
            if tol is None:
                solver.advance(goal)
                solver.synchronize()
            else:
                converged_time = _advance_until(solver, goal, tol)
            update_seconds += time.perf_counter() - t0
            frames += 1
            kept_times.append(float(solver.time if converged_time else goal))
            if writer:
                writer.submit()
            save_probes()
            if index % 5 == 0 or index == len(times) - 1 or converged_time:
                resolved = int(np.isfinite(solver.arrival()).sum())
                row = dict(time=kept_times[-1], steps=solver.steps,
                           resolved=resolved,
                           elapsed_seconds=time.perf_counter() - started)
                progress.write(json.dumps(row) + "\n")
                progress.flush()
                log.write(f"budget={row['time']} steps={row['steps']} "
                          f"resolved={resolved} elapsed={row['elapsed_seconds']}\n")
                log.flush()
            if converged_time is not None:
                break
    finally:
        try:
            if writer:
                writer.close()
                transfer_seconds, write_seconds = writer.transfer_seconds, writer.write_seconds
        finally:
            if history_file:
                history_file.close()
            if probe_file:
                probe_file.close()
            log.close()
            progress.close()
    final_write = 0.0
    if save_final:
        t0 = time.perf_counter()
        solver.field(host).tofile(output / "final.f32")
        solver.arrival(host).tofile(output / "arrival.f32")
        final_write = time.perf_counter() - t0
    residual, increase = solver.stats()
    timing = {
        "states": N,
        "working_array_bytes": 12 * N,
        "cfl_dt_limit": solver.cfl_dt_limit,
        "internal_steps": solver.steps,
        "frames": frames,
        "update_seconds": update_seconds,
        "device_to_host_seconds": transfer_seconds,
        "history_write_seconds": write_seconds,
        "final_write_seconds": final_write,
        "probe_seconds": probe_seconds,
        "elapsed_seconds": time.perf_counter() - started,
        "maximum_increase": increase,
        "last_step_residual": residual,
        "cell_backups_per_second":
            N * solver.steps * (2 if _order(solver) == 2 else 1)
            / max(update_seconds, 1e-12),
    }
    (output / "timing.json").write_text(json.dumps(timing) + "\n")
    result = dict(timing)
    result["times"] = kept_times
    if converged_time is not None:
        result["converged_time"] = converged_time
    return result


def _order(solver):
    return solver._params.order


def _advance_until(solver, goal, tol):
    """Step toward `goal`; return the time at which a step's sup-norm change
    fell below tol, or None if it did not before `goal`."""
    limit = solver.cfl_dt_limit
    while solver.time < goal - 1e-12:
        solver.step(min(limit, goal - solver.time))
        residual, _ = solver.stats()
        if residual < tol:
            return solver.time
    return None


def main():
    import argparse
    from .model import ReversibleConfig

    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("output")
    parser.add_argument("--config")
    parser.add_argument("--positions", type=int, default=41)
    parser.add_argument("--headings", type=int, default=24)
    parser.add_argument("--p-speeds", type=int, default=7)
    parser.add_argument("--e-speeds", type=int, default=7)
    parser.add_argument("--extent", type=float, default=4)
    parser.add_argument("--horizon", type=float, default=2)
    parser.add_argument("--output-dt", type=float, default=0.1)
    parser.add_argument("--threads", type=int, default=4)
    parser.add_argument("--order", type=int, choices=[1, 2], default=2)
    parser.add_argument("--no-history", action="store_true")
    parser.add_argument("--max-working-gb", type=float, default=8)
    parser.add_argument("--local-precision", choices=["float32", "float64"],
                        default="float64")
    parser.add_argument("--tol", type=float)
    args = parser.parse_args()
    config = (
        ReversibleConfig.from_dict(json.loads(Path(args.config).read_text()))
        if args.config else ReversibleConfig()
    )
    grid = RelativeGrid(args.positions, args.headings, args.p_speeds,
                        args.e_speeds, args.extent)
    result = solve(config, grid, args.output, horizon=args.horizon,
                   output_dt=args.output_dt, threads=args.threads,
                   order=args.order, history=not args.no_history,
                   max_working_gb=args.max_working_gb,
                   local_precision=args.local_precision, tol=args.tol)
    print(json.dumps({k: result[k] for k in
                      ("status", "states", "update_seconds",
                       "cell_backups_per_second")}, indent=2))


if __name__ == "__main__":
    main()
