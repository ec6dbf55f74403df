"""The legacy 6D square solver on the GPU (replaces
src/pursuit_evasion/dp/native.py:14-106, which compiles and runs the
executable native_square.cpp).  Same signature, output folder and metadata:
meta.json, fields.f32 (every output frame, float32 [T, xP, yP, thP, xE, yE,
thE]), final.f32, arrival.f32, native_timing.json and solver.log; the
fields equal the executable's bit for bit (csrc/square6d_exact.cu)."""

from __future__ import annotations

import ctypes
import json
from pathlib import Path
import time

import numpy as np

from .. import _native
from ..model import GameConfig
from .grid import GridSpec, output_times
from .options import validate_options


def _params(config: GameConfig, grid: GridSpec, *, order, cfl, device):
    return _native.SquareParams(
        positions=int(grid.positions), headings=int(grid.headings),
        extent=float(grid.extent), arena=float(config.arena_half_width),
        capture_radius=float(config.capture_radius),
        p_speed=float(config.pursuer.speed), e_speed=float(config.evader.speed),
        p_turn_rate=float(config.pursuer.max_turn_rate),
        e_turn_rate=float(config.evader.max_turn_rate),
        cfl=float(cfl), order=int(order), device=int(device))


class SquareSolver:
    """GPU handle of the 6D square game (pe_square_*)."""

    def __init__(self, config: GameConfig, grid: GridSpec, *, order=2, cfl=0.8, device=0):
        self._lib = _native.library()
        self.grid = grid
        self.shape = tuple(grid.shape)
        self.cells = grid.states
        self._params = _params(config, grid, order=order, cfl=cfl, device=device)
        handle = ctypes.c_void_p()
        _native.check(self._lib.pe_square_create(ctypes.byref(self._params),
                                                 ctypes.byref(handle)))
        self._h = handle
        dt = ctypes.c_double()
        _native.check(self._lib.pe_square_dt_limit(ctypes.byref(self._params),
                                                    ctypes.byref(dt)))
        self.dt_limit = dt.value

    def close(self):
        if getattr(self, "_h", None):
            _native.check(self._lib.pe_square_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def initialize(self):
        _native.check(self._lib.pe_square_init(self._h))

    def advance(self, goal):
        steps = ctypes.c_int64()
        _native.check(self._lib.pe_square_advance(self._h, float(goal), ctypes.byref(steps)))
        return steps.value

    @property
    def time(self):
        t, n = ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.pe_square_time(self._h, ctypes.byref(t), ctypes.byref(n)))
        return t.value

    @property
    def steps(self):
        t, n = ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.pe_square_time(self._h, ctypes.byref(t), ctypes.byref(n)))
        return n.value

    def synchronize(self):
        _native.check(self._lib.pe_square_synchronize(self._h))

    def field(self, out=None):
        out = np.empty(self.cells, np.float32) if out is None else out
        _native.check(self._lib.pe_square_copy_field(self._h, out.ctypes.data))
        return out.reshape(self.shape)

    def arrival(self, out=None):
        out = np.empty(self.cells, np.float32) if out is None else out
        _native.check(self._lib.pe_square_copy_arrival(self._h, out.ctypes.data))
        return out.reshape(self.shape)

    def residual(self):
        r = ctypes.c_double()
        _native.check(self._lib.pe_square_residual(self._h, ctypes.byref(r)))
        return r.value

    def profile(self, enable=True):
        _native.check(self._lib.pe_square_profile(self._h, int(enable)))

    def kernel_time(self):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.pe_square_kernel_time(self._h, ctypes.byref(ms),
                                                      ctypes.byref(n)))
        return ms.value, n.value


def solve(config: GameConfig, grid: GridSpec, output, *, horizon=2.0, output_dt=0.1,
          order=2, cfl=0.8, threads=8, history=True, device=0):
    """The reference's dp.native.solve: validate, write meta.json, run the
    frame loop of native_square.cpp:185-202 (here on the GPU) and save the
    fields; `threads` is accepted and recorded (the work runs on the GPU)."""
    validate_options(horizon, output_dt, order, cfl, threads)
    output = Path(output).resolve()
    if (output / "meta.json").exists():
        raise FileExistsError(f"Preserve completed solve: {output}")
    output.mkdir(parents=True, exist_ok=True)
    times = output_times(horizon, output_dt)
    meta = dict(
        backend="b200_cuda", config=config.to_dict(), grid=grid.to_dict(), horizon=horizon,
        output_dt=output_dt, times=times.tolist(), order=order, cfl=cfl, threads=threads,
        history_saved=history, dtype="float32", compile_seconds=0.0,
        target="capture_or_evader_boundary_fault", avoid="pursuer_boundary_fault",
        tube_projection="min over every internal update, then max with avoid",
        status="running")
    (output / "meta.json").write_text(json.dumps(meta, indent=2) + "\n")
    started = time.perf_counter()
    status = "failed"
    try:
        with SquareSolver(config, grid, order=order, cfl=cfl, device=device) as s, \
                (output / "solver.log").open("w") as log:
            t0 = time.perf_counter()
            s.initialize()
            init_seconds = time.perf_counter() - t0
            update_seconds = write_seconds = 0.0
            host = np.empty(s.cells, np.float32)
            frames = 0
            fields = (output / "fields.f32").open("wb") if history else None
            try:
                def save():
                    nonlocal write_seconds, frames
                    t = time.perf_counter()
                    if fields:
                        s.field(host).tofile(fields)
                    write_seconds += time.perf_counter() - t
                    frames += 1

                save()
                for frame in range(1, int(np.ceil(horizon / output_dt - 1e-10)) + 1):
                    goal = min(horizon, frame * output_dt)
                    t = time.perf_counter()
                    s.advance(goal)
                    s.synchronize()
                    update_seconds += time.perf_counter() - t
                    save()
                    log.write(f"budget {s.time} steps {s.steps} updates_s {update_seconds}\n")
            finally:
                if fields:
                    fields.close()
            t = time.perf_counter()
            s.field(host).tofile(output / "final.f32")
            s.arrival(host).tofile(output / "arrival.f32")
            write_seconds += time.perf_counter() - t
            timing = dict(states=s.cells, internal_steps=s.steps, frames=frames,
                          update_seconds=update_seconds, initialization_seconds=init_seconds,
                          write_seconds=write_seconds,
                          process_seconds=time.perf_counter() - started,
                          core_array_bytes=s.cells * 12, max_internal_dt=s.dt_limit,
                          arithmetic="float32 fields and float32 local arithmetic")
            (output / "native_timing.json").write_text(json.dumps(timing) + "\n")
            status = "complete"
    finally:
        meta.update(subprocess_seconds=time.perf_counter() - started, status=status)
        if status == "complete":
            meta.update(timing)
        (output / "meta.json").write_text(json.dumps(meta, indent=2) + "\n")
    return meta
