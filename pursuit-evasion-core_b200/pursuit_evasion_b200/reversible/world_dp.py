"""Dense 8D reversible-car game on B200: the ENO/Lax-Friedrichs HJI step.

Mirrors pursuit-evasion-core src/pursuit_evasion/reversible/world_dp.py
(WorldGrid :24-97, global_rate_bound :101-113, solve :177-463) for the
square-arena game, with the per-cell work in hand-written sm_100a kernels
behind libpe_b200.so (pe_world_* C ABI) instead of the g++/OpenMP
executable native_world.cpp.  Arithmetic is float32 in the reference's
order; results equal the executable's bit for bit.

Two capture fields:
  * "square" — the reference's capture-or-E-fault target with the P-fault
    avoid floor (native_world.cpp:155-176);
  * "contact" — the 8D contact game: exact oriented-rectangle contact of
    the two footprints (separating axes, local_game/geometry.py:15-36) and
    no avoid floor.
"""

from __future__ import annotations

import ctypes
from dataclasses import asdict, dataclass
import json
import math
from pathlib import Path
import time

import numpy as np

from .. import _native
from .model import config_dict

STATE_ORDER = ["xP", "yP", "thetaP", "vP", "xE", "yE", "thetaE", "vE"]
PERIODIC_AXES = (2, 6)


@dataclass(frozen=True)
class WorldGrid:
    positions: int = 9
    headings: int = 8
    p_speeds: int = 7
    e_speeds: int = 7
    extent: float = 3.5

    def __post_init__(self):
        for name, minimum in [("positions", 5), ("headings", 4), ("p_speeds", 3),
                              ("e_speeds", 3)]:
            value = getattr(self, name)
            if (isinstance(value, bool) or not isinstance(value, (int, np.integer))
                    or value < minimum):
                raise ValueError(f"{name} must be an integer >= {minimum}.")
        if not np.isfinite(self.extent) or self.extent <= 0:
            raise ValueError("extent must be finite and positive.")

    @property
    def shape(self):
        n, h = self.positions, self.headings
        return (n, n, h, self.p_speeds, n, n, h, self.e_speeds)

    @property
    def states(self):
        return math.prod(self.shape)

    def axes(self, config):
        x = np.linspace(-self.extent, self.extent, self.positions)
        theta = -np.pi + np.arange(self.headings) * 2 * np.pi / self.headings
        vp = np.linspace(config.pursuer.speed_min, config.pursuer.speed_max,
                         self.p_speeds)
        ve = np.linspace(config.evader.speed_min, config.evader.speed_max,
                         self.e_speeds)
        return (x, x, theta, vp, x, x, theta, ve)

    def to_dict(self):
        return asdict(self)


def global_rate_bound(config, grid):
    """Sum of rate/spacing over the axes (world_dp.py:101-113)."""
    dx, _, dh, dvp, _, _, _, dve = [float(a[1] - a[0]) for a in grid.axes(config)]
    p, e = config.pursuer, config.evader
    vp = max(abs(p.speed_min), abs(p.speed_max))
    ve = max(abs(e.speed_min), abs(e.speed_max))
    return (2 * (vp + ve) / dx + (vp * p.max_curvature + ve * e.max_curvature) / dh
            + p.acceleration / dvp + e.acceleration / dve)


def output_times(horizon, output_dt):
    if not np.isfinite([horizon, output_dt]).all() or min(horizon, output_dt) <= 0:
        raise ValueError("Positive finite horizon and output_dt are required.")
    return np.unique(np.minimum(
        np.arange(int(np.ceil(horizon / output_dt)) + 1) * output_dt, horizon))


def _params(config, grid, *, order, cfl, speed_boundary, avoid, device, fast=False):
    p, e = config.pursuer, config.evader
    return _native.WorldParams(
        positions=grid.positions, headings=grid.headings,
        p_speeds=grid.p_speeds, e_speeds=grid.e_speeds,
        extent=float(grid.extent), arena=float(config.arena_half_width),
        capture_radius=float(config.capture_radius),
        p_speed_min=float(p.speed_min), p_speed_max=float(p.speed_max),
        p_acceleration=float(p.acceleration), p_curvature=float(p.max_curvature),
        e_speed_min=float(e.speed_min), e_speed_max=float(e.speed_max),
        e_acceleration=float(e.acceleration), e_curvature=float(e.max_curvature),
        cfl=float(cfl), order=int(order),
        linear_speed_boundary=int(speed_boundary == "linear"),
        avoid_mode={False: 0, None: 0, True: 1, "square": 1, "clearance": 2}[avoid],
        device=int(device), fast=int(bool(fast)))


class WorldSolver:
    """Owning handle of one device-resident 8D field (pe_world_*).  `fast`
    selects the stage with reciprocal spacings and multiply-add contraction
    instead of the reference's operation order (bit for bit
    native_world.cpp).  `avoid`: True (or "square") for the square-arena
    floor, False for none, "clearance" for the obstacle map game's floor
    -p_clear + 1e-6 (gpu_map_game.py:64-66; set_clearance first)."""

    def __init__(self, config, grid, *, order=2, cfl=0.8, speed_boundary="linear",
                 avoid=True, device=0, fast=False):
        if speed_boundary not in ("linear", "legacy_signed"):
            raise ValueError("Speed boundary must be linear or legacy_signed.")
        if order not in (1, 2) or not 0 < cfl <= 1:
            raise ValueError("Require order 1/2 and CFL in (0, 1].")
        self._lib = _native.library()
        self.grid = grid
        self.shape = grid.shape
        self.cells = grid.states
        self._params = _params(config, grid, order=order, cfl=cfl,
                               speed_boundary=speed_boundary, avoid=avoid,
                               device=device, fast=fast)
        handle = ctypes.c_void_p()
        _native.check(self._lib.pe_world_create(ctypes.byref(self._params),
                                                ctypes.byref(handle)))
        self._h = handle
        dt = ctypes.c_double()
        _native.check(self._lib.pe_world_dt_limit(ctypes.byref(self._params),
                                                  ctypes.byref(dt)))
        self.dt_limit = dt.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pe_world_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def init_contact(self, p_footprint, e_footprint):
        """p/e footprints as (length, width)."""
        _native.check(self._lib.pe_world_init_contact(
            self._h, float(p_footprint[0]), float(p_footprint[1]),
            float(e_footprint[0]), float(e_footprint[1])))

    def init_square(self):
        _native.check(self._lib.pe_world_init_square(self._h))

    def set_clearance(self, p_clear, e_clear):
        """Each car's obstacle clearance per (x, y, heading) grid pose,
        [positions, positions, headings] (FootprintMap.clearance at the grid
        poses, gpu_map_game.py:78-84)."""
        n, nh = self.grid.positions, self.grid.headings
        arrays = [np.ascontiguousarray(c, dtype=np.float32) for c in (p_clear, e_clear)]
        for c in arrays:
            if c.shape != (n, n, nh):
                raise ValueError("clearance grids must be [positions, positions, headings]")
        _native.check(self._lib.pe_world_set_clearance(self._h, arrays[0].ctypes.data,
                                                       arrays[1].ctypes.data))

    def init_map(self):
        """The map game's surfaces (gpu_map_game.py:45-50): max(min(centre
        distance - radius, e_clear), -p_clear + 1e-6)."""
        _native.check(self._lib.pe_world_init_map(self._h))

    def init_field(self, field, arrival=None, start_time=0.0):
        field = np.ascontiguousarray(field, dtype=np.float32).reshape(-1)
        if field.size != self.cells:
            raise ValueError("field has the wrong number of cells")
        arr_ptr = None
        if arrival is not None:
            arrival = np.ascontiguousarray(arrival, dtype=np.float32).reshape(-1)
            arr_ptr = arrival.ctypes.data
        _native.check(self._lib.pe_world_init_field(self._h, field.ctypes.data,
                                                    arr_ptr, float(start_time)))

    def advance(self, goal):
        steps = ctypes.c_int64()
        _native.check(self._lib.pe_world_advance(self._h, float(goal),
                                                 ctypes.byref(steps)))
        return steps.value

    def step(self, dt):
        _native.check(self._lib.pe_world_step(self._h, float(dt)))

    @property
    def time(self):
        t, n = ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.pe_world_time(self._h, ctypes.byref(t), ctypes.byref(n)))
        return t.value

    @property
    def steps(self):
        t, n = ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.pe_world_time(self._h, ctypes.byref(t), ctypes.byref(n)))
        return n.value

    def synchronize(self):
        _native.check(self._lib.pe_world_synchronize(self._h))

    def field(self, out=None):
        out = np.empty(self.cells, np.float32) if out is None else out
        _native.check(self._lib.pe_world_copy_field(self._h, out.ctypes.data))
        return out.reshape(self.shape)

    def arrival(self, out=None):
        out = np.empty(self.cells, np.float32) if out is None else out
        _native.check(self._lib.pe_world_copy_arrival(self._h, out.ctypes.data))
        return out.reshape(self.shape)

    def residual(self):
        r = ctypes.c_double()
        _native.check(self._lib.pe_world_residual(self._h, ctypes.byref(r)))
        return r.value

    def set_stream(self, stream_ptr):
        _native.check(self._lib.pe_world_set_stream(self._h, stream_ptr))

    def profile(self, enable=True):
        _native.check(self._lib.pe_world_profile(self._h, int(enable)))

    def kernel_time(self):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.pe_world_kernel_time(self._h, ctypes.byref(ms),
                                                     ctypes.byref(n)))
        return ms.value, n.value


def solve(config, grid, output, *, horizon=0.5, output_dt=0.25, order=2, cfl=0.8,
          threads=8, history=False, max_core_gb=12.0, max_output_gb=30.0,
          speed_boundary="linear", write_final=True, write_arrival=True,
          capture_footprints=None, device=0):
    """Solve the 8D game on the GPU and write a table directory.

    Same guards and files as world_dp.py:177-463 (meta.json, fields.f32 when
    history is kept, final.f32, arrival.f32).  capture_footprints=(P, E), each
    (length, width), selects the contact game (rectangle-contact capture, no
    avoid floor); otherwise the reference's square-arena surfaces are used.
    """
    if grid.extent <= config.arena_half_width and capture_footprints is None:
        raise ValueError("Numerical domain must include exterior padding.")
    if speed_boundary not in ("linear", "legacy_signed"):
        raise ValueError("Speed boundary must be linear or legacy_signed.")
    if order not in (1, 2) or not 0 < cfl <= 1 or not isinstance(threads, int) or threads < 1:
        raise ValueError("Require order1/2, CFL in(0,1], positive integer threads.")
    if not history and not write_final:
        raise ValueError("Retain history or a final field.")
    times = output_times(horizon, output_dt)
    core_bytes = grid.states * 12
    output_bytes = grid.states * 4 * (int(write_final) + int(write_arrival)
                                      + (len(times) if history else 0))
    if (not np.isfinite([max_core_gb, max_output_gb]).all()
            or min(max_core_gb, max_output_gb) <= 0):
        raise ValueError("Positive explicit resource limits are required.")
    if core_bytes > max_core_gb * 1e9 or output_bytes > max_output_gb * 1e9:
        raise MemoryError(f"Requested core {core_bytes / 1e9:.3f}GB, outputs "
                          f"{output_bytes / 1e9:.3f}GB exceed limits.")
    output = Path(output).resolve()
    if (output / "meta.json").exists():
        raise FileExistsError(f"Preserve existing run: {output}")
    started = time.perf_counter()
    contact = capture_footprints is not None
    solver = WorldSolver(config, grid, order=order, cfl=cfl,
                         speed_boundary=speed_boundary, avoid=not contact,
                         device=device)
    output.mkdir(parents=True, exist_ok=True)
    meta = dict(schema="reversible_world8d_v1", backend="b200_cuda_world8d",
                status="running", config=config_dict(config), grid=grid.to_dict(),
                shape=list(grid.shape), state_order=STATE_ORDER,
                axes=[a.tolist() for a in grid.axes(config)], times=times.tolist(),
                horizon=horizon, output_dt=output_dt, order=order, cfl=cfl,
                speed_boundary=speed_boundary, history_saved=bool(history),
                capture=("rectangle_contact" if contact else "square_arena"),
                capture_footprints=(None if not contact else
                                    [list(map(float, f)) for f in capture_footprints]),
                avoid=None if contact else "pursuer_square_fault",
                dtype="float32", max_internal_dt=solver.dt_limit)
    (output / "meta.json").write_text(json.dumps(meta, indent=2))
    try:
        if contact:
            solver.init_contact(*capture_footprints)
        else:
            solver.init_square()
        host = np.empty(grid.states, np.float32)
        history_file = (output / "fields.f32").open("wb") if history else None
        update_seconds = 0.0
        try:
            if history_file:
                solver.field(host).tofile(history_file)
            for goal in times[1:]:
                t0 = time.perf_counter()
                solver.advance(goal)
                solver.synchronize()
                update_seconds += time.perf_counter() - t0
                if history_file:
                    solver.field(host).tofile(history_file)
        finally:
            if history_file:
                history_file.close()
        if write_final:
            solver.field(host).tofile(output / "final.f32")
        if write_arrival:
            solver.arrival(host).tofile(output / "arrival.f32")
        meta.update(status="complete", internal_steps=solver.steps,
                    update_seconds=update_seconds, states=grid.states,
                    wall_seconds=time.perf_counter() - started,
                    cell_backups_per_second=grid.states * solver.steps * order
                    / max(update_seconds, 1e-12))
    except Exception as exc:
        meta.update(status="failed", failure=str(exc))
        raise
    finally:
        solver.close()
        (output / "meta.json").write_text(json.dumps(meta, indent=2))
    return meta
