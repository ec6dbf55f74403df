"""Batched relative 5D solves (pe_batch_*): many free_dp-style solves of
different grid sizes, physics and horizons in one persistent launch.

`BatchSolver` owns the device fields of every solve; `run()` advances all of
them to their horizons with one CUDA-graph launch of one cooperative kernel.
With the exact arithmetic each solve's result equals a float64
`RelativeSolver` advanced to the same horizon (and the reference
executable's), bit for bit; the float32 cell update is the fast variant.
`draw_batch` draws the heterogeneous solve set of the batched workload from
a seed; `autotune.tune` picks the work-item tile per size bucket.  The
solves are independent, so several GPUs split a batch with `partition`
(each rank builds a `BatchSolver` on its own share, `local_share`) and
exchange nothing.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, replace

import numpy as np

from .. import _native
from ..reversible.free_dp import RelativeGrid
from ..reversible.model import ReversibleConfig, VehicleLimits
from ..reversible.relative_solver import _params, cfl_limit


@dataclass(frozen=True)
class BatchSolve:
    config: ReversibleConfig
    grid: RelativeGrid
    horizon: float


def draw_batch(seed, count=256, *, extent=4.0, base=None):
    """The heterogeneous solve set: per solve, positions ~U{17..49}, headings
    ~U{12..36}, speeds ~U{7..15} per car, acceleration ~U(1.5, 4) per car,
    capture radius ~U(0.3, 0.8) and horizon ~U(0.5, 2) s, drawn with
    numpy.random.default_rng(seed); the other limits from `base` (the a3
    physics by default) and the position box [-extent, extent]^2."""
    if base is None:
        base = ReversibleConfig(name="reversible_free_a3",
                                pursuer=VehicleLimits(-1.0, 2.0, 3.0, 1.0),
                                evader=VehicleLimits(-0.5, 1.0, 3.0, 2.0))
    rng = np.random.default_rng(seed)
    solves = []
    for _ in range(count):
        positions = int(rng.integers(17, 50))
        headings = int(rng.integers(12, 37))
        p_speeds = int(rng.integers(7, 16))
        e_speeds = int(rng.integers(7, 16))
        acc_p = float(rng.uniform(1.5, 4.0))
        acc_e = float(rng.uniform(1.5, 4.0))
        radius = float(rng.uniform(0.3, 0.8))
        horizon = float(rng.uniform(0.5, 2.0))
        config = replace(base, name=f"{base.name}_batch",
                         pursuer=replace(base.pursuer, acceleration=acc_p),
                         evader=replace(base.evader, acceleration=acc_e),
                         capture_radius=radius)
        grid = RelativeGrid(positions, headings, p_speeds, e_speeds, float(extent))
        solves.append(BatchSolve(config, grid, horizon))
    return solves


def describe(solves):
    """JSON-ready table of a solve set."""
    return [dict(positions=s.grid.positions, headings=s.grid.headings,
                 p_speeds=s.grid.p_speeds, e_speeds=s.grid.e_speeds,
                 extent=s.grid.extent, p_acceleration=s.config.pursuer.acceleration,
                 e_acceleration=s.config.evader.acceleration,
                 capture_radius=s.config.capture_radius, horizon=s.horizon)
            for s in solves]


def solve_steps(solve, *, cfl=0.8):
    """RK2 steps of one solve to its horizon: steps of the CFL limit, the
    last one cut to the horizon (the schedule of pe_batch_create)."""
    limit = cfl_limit(solve.config, solve.grid, cfl=cfl)
    t, steps = 0.0, 0
    while t < solve.horizon - 1e-12:
        t += min(limit, solve.horizon - t)
        steps += 1
    return steps


def solve_work(solve, *, cfl=0.8):
    """Cell-stages of one solve: cells x 2 stages x RK2 steps."""
    return solve.grid.states * 2 * solve_steps(solve, cfl=cfl)


def partition(solves, parts, *, cfl=0.8):
    """Split a batch over `parts` GPUs: a list of `parts` sorted index
    lists that together hold every solve once.  Greedy longest first: the
    solves in decreasing cell-stages (ties by index) each go to the share
    with the least work so far (ties to the lowest share), so every share
    ends within one solve's work of the mean.  The result depends only on
    the solves, so every rank computes the same split without talking."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    work = [solve_work(s, cfl=cfl) for s in solves]
    order = sorted(range(len(solves)), key=lambda i: (-work[i], i))
    load = [0] * parts
    shares = [[] for _ in range(parts)]
    for i in order:
        k = min(range(parts), key=lambda j: (load[j], j))
        shares[k].append(i)
        load[k] += work[i]
    return [sorted(sh) for sh in shares]


def local_share(solves, rank, world, *, cfl=0.8):
    """(indices, solves) of rank `rank` of `world` under `partition`."""
    if not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    idx = partition(solves, world, cfl=cfl)[rank]
    return idx, [solves[i] for i in idx]


class BatchSolver:
    """`local_precision`: "float64" (the exact arithmetic: each solve equals a
    float64 RelativeSolver bit for bit) or "float32" (the float32 cell
    update)."""

    def __init__(self, solves, *, cfl=0.8, local_precision="float64", device=0):
        if local_precision not in ("float32", "float64"):
            raise ValueError("local_precision must be 'float32' or 'float64'")
        self._lib = _native.library()
        self.solves = list(solves)
        self.local_precision = local_precision
        count = len(self.solves)
        precision = (_native.PE_LOCAL_F64 if local_precision == "float64"
                     else _native.PE_LOCAL_F32)
        params = (_native.RelativeParams * count)(*[
            _params(s.config, s.grid, order=2, cfl=cfl, precision=precision,
                    device=device) for s in self.solves])
        horizons = (ctypes.c_double * count)(*[float(s.horizon) for s in self.solves])
        handle = ctypes.c_void_p()
        _native.check(self._lib.pe_batch_create(params, horizons, count, int(device),
                                                ctypes.byref(handle)))
        self._h = handle

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pe_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self.solves)

    def set_tile(self, solve, rows):
        _native.check(self._lib.pe_batch_set_tile(self._h, int(solve), int(rows)))

    def tile(self, solve):
        r = ctypes.c_int32()
        _native.check(self._lib.pe_batch_get_tile(self._h, int(solve), ctypes.byref(r)))
        return r.value

    def set_stream(self, stream_ptr):
        _native.check(self._lib.pe_batch_set_stream(self._h, stream_ptr))

    def initialize(self):
        _native.check(self._lib.pe_batch_init(self._h))

    def run(self):
        _native.check(self._lib.pe_batch_run(self._h))

    def synchronize(self):
        _native.check(self._lib.pe_batch_synchronize(self._h))

    def info(self, solve):
        cells, steps, limit = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
        _native.check(self._lib.pe_batch_solve_info(self._h, int(solve), ctypes.byref(cells),
                                                    ctypes.byref(steps), ctypes.byref(limit)))
        return dict(cells=cells.value, steps=steps.value, dt_limit=limit.value)

    def launch_info(self):
        ctas, threads, steps = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        total = ctypes.c_int64()
        _native.check(self._lib.pe_batch_launch_info(
            self._h, ctypes.byref(ctas), ctypes.byref(threads), ctypes.byref(steps),
            ctypes.byref(total)))
        return dict(ctas=ctas.value, threads=threads.value, max_steps=steps.value,
                    cell_stages=total.value)

    def field(self, solve):
        g = self.solves[solve].grid
        out = np.empty(g.states, np.float32)
        _native.check(self._lib.pe_batch_copy_field(self._h, int(solve), out.ctypes.data))
        return out.reshape(g.shape)

    def arrival(self, solve):
        g = self.solves[solve].grid
        out = np.empty(g.states, np.float32)
        _native.check(self._lib.pe_batch_copy_arrival(self._h, int(solve), out.ctypes.data))
        return out.reshape(g.shape)

    def stats(self, solve):
        r, inc = ctypes.c_double(), ctypes.c_double()
        _native.check(self._lib.pe_batch_stats(self._h, int(solve), ctypes.byref(r),
                                               ctypes.byref(inc)))
        return r.value, inc.value

    def profile(self, enable=True):
        _native.check(self._lib.pe_batch_profile(self._h, int(enable)))

    def kernel_time(self):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.pe_batch_kernel_time(self._h, ctypes.byref(ms),
                                                     ctypes.byref(n)))
        return ms.value, n.value
