"""The 8D obstacle map game (the reference's reversible/gpu_map_game.py) on
the pe_world_* solver: center-distance capture, first-fault-loses, each
car's clearance to the obstacles per (x, y, heading) grid pose.  The signed
field is a pursuer-success reach-avoid value, not a capture time.

Same entry points, arguments, errors and output folder as the reference
(`solve`, `clearance_grids`, `node_states`; meta.json, labels.npz,
optional fields.f32 / final.f32, progress.jsonl).  `geometry` is any object
with the reference FootprintMap's `clearance(poses, role)` and `to_dict()`
(the reference's FootprintMap itself), or a (p_clear, e_clear) pair of
[positions, positions, headings] arrays.
"""

from __future__ import annotations

from itertools import product
import json
from pathlib import Path
import shutil
import time

import numpy as np

from .world_dp import WorldGrid, WorldSolver, output_times


def clearance_grids(geometry, grid, config):
    """Each car's clearance at every (x, y, heading) grid pose
    (gpu_map_game.py:78-84)."""
    axes = grid.axes(config)
    x, y, h = np.meshgrid(axes[0], axes[1], axes[2], indexing="ij")
    poses = np.stack([x, y, h], axis=-1)
    return tuple(np.asarray(geometry.clearance(poses, role), np.float32)
                 for role in ("pursuer", "evader"))


def node_states(indices, grid, config):
    """Grid states of flat node indices (gpu_map_game.py:87-89)."""
    q = np.unravel_index(np.asarray(indices, np.int64), grid.shape)
    return np.stack([axis[i] for axis, i in zip(grid.axes(config), q)], axis=-1)


def interpolation_stencil(states, axes, periodic_axes):
    """2^d-corner multilinear stencils over the flat storage order
    (world_table.py:13-45): periodic axes wrap, the others clamp to the last
    interval; returns (indices, weights, valid)."""
    s = np.asarray(states, dtype=float)
    d = len(axes)
    flat = s.reshape(-1, d)
    valid = np.isfinite(flat).all(1)
    safe = np.where(np.isfinite(flat), flat, 0.0)
    shape = tuple(len(a) for a in axes)
    stride = np.ones(d, np.int64)
    for k in range(d - 2, -1, -1):
        stride[k] = stride[k + 1] * shape[k + 1]
    corner = (np.arange(2 ** d)[:, None] >> np.arange(d - 1, -1, -1)[None, :]) & 1
    indices = np.zeros((len(flat), 2 ** d), np.int64)
    weights = np.ones((len(flat), 2 ** d))
    for k, axis in enumerate(axes):
        axis = np.asarray(axis, float)
        n, h = len(axis), float(axis[1] - axis[0])
        q = safe[:, k]
        if k in periodic_axes:
            f = np.mod(q - axis[0], h * n) / h
            low = np.floor(f).astype(np.int64) % n
            w = f - np.floor(f)
        else:
            valid &= (q >= axis[0] - 1e-10) & (q <= axis[-1] + 1e-10)
            f = (np.clip(q, axis[0], axis[-1]) - axis[0]) / h
            low = np.minimum(np.floor(f).astype(np.int64), n - 2)
            w = np.clip(f - low, 0, 1)
        node = low[:, None] + corner[None, :, k]
        if k in periodic_axes:
            node %= n
        indices += node * stride[k]
        weights *= np.where(corner[None, :, k] == 1, w[:, None], 1 - w[:, None])
    return indices, weights, valid


def solve(config, grid, geometry, output, *, horizon=1.5, output_dt=0.5, order=2, cfl=0.7,
          query_indices=None, query_states=None, save_final=False, save_history=False,
          max_working_gb=7.6, device=0, fast=False):
    """Solve the map game and sample the field at the query nodes or states
    after every output interval (gpu_map_game.py:92-303).  `fast` selects
    the float32 stage with multiply-add contraction."""
    if config.capture_rule != "center_distance" or config.boundary_rule != "first_fault_loses":
        raise ValueError("Legacy map HJI uses center-distance capture and first-fault-loses")
    if config.point_vehicles:
        raise ValueError("Footprint HJI requires point_vehicles=False.")
    pair = isinstance(geometry, (tuple, list)) and len(geometry) == 2
    if not isinstance(grid, WorldGrid) or not (pair or hasattr(geometry, "clearance")):
        raise TypeError("Use explicit FootprintMap (or clearance grids) and WorldGrid")
    half_width = None if pair else getattr(geometry, "half_width", None)
    if order not in (1, 2) or not 0 < cfl <= 1 or (
            half_width is not None and grid.extent <= half_width):
        raise ValueError("Require order1/2, CFL<=1 and spatial exterior padding")
    output = Path(output)
    output.mkdir(parents=True, exist_ok=True)
    if (output / "meta.json").exists():
        raise FileExistsError("Preserve existing solve")
    n = grid.states
    working = n * 12
    if working > max_working_gb * 1e9:
        raise MemoryError(f"Need {working / 1e9:.3f} GB core GPU arrays")
    idx = np.asarray([] if query_indices is None else query_indices, np.int64)
    if idx.ndim != 1 or ((idx < 0) | (idx >= n)).any():
        raise ValueError("Invalid query node indices")
    stencil = weights = None
    states = node_states(idx, grid, config)
    if query_states is not None:
        if query_indices is not None:
            raise ValueError("Choose node indices OR continuous query states")
        states = np.asarray(query_states, float)
        if states.ndim != 2 or states.shape[1] != 8 or len(states) > 100000:
            raise ValueError("Expected at most100000 world states[n,8]")
        stencil, weights, valid = interpolation_stencil(states, grid.axes(config), (2, 6))
        if not valid.all():
            raise ValueError("Query outside numerical domain")
    times = output_times(horizon, output_dt)
    expected = 4 * n * (int(save_final) + len(times) * int(save_history))
    if shutil.disk_usage(output).free < expected + 5 * 10 ** 9:
        raise OSError("Insufficient disk space for requested retained fields")
    pc, ec = (tuple(np.asarray(c, np.float32) for c in geometry) if pair
              else clearance_grids(geometry, grid, config))
    started = time.perf_counter()
    meta = dict(
        schema="footprint_map_game8d_v1",
        status="running",
        backend="b200_cuda",
        config=config.to_dict(),
        geometry=None if pair else geometry.to_dict(),
        grid=grid.to_dict(),
        times=times.tolist(),
        target="capture_OR_evader_collision",
        avoid="pursuer_collision",
        game_rule="first_fault_loses; P collision wins numerical event ties",
        output_meaning="signed finite-budget P-success reach-avoid value, NOT capture time",
        core_array_bytes=working,
        order=order,
        cfl=cfl,
        local_precision="float32",
        stage="fast" if fast else "reference_order",
        state_order=["xP", "yP", "headingP", "vP", "xE", "yE", "headingE", "vE"],
        query_count=len(states),
        history_saved=bool(save_history),
    )
    (output / "meta.json").write_text(json.dumps(meta, indent=2))
    host = np.empty(n, np.float32)
    with WorldSolver(config, grid, order=order, cfl=cfl, speed_boundary="linear",
                     avoid="clearance", device=device, fast=fast) as s:
        s.set_clearance(pc, ec)
        s.init_map()

        def sample():
            s.field(host)
            return host[idx] if weights is None else (host[stencil] * weights).sum(axis=1)

        history = (output / "fields.f32").open("wb") if save_history else None
        try:
            samples = [sample()]
            if history is not None:
                host.tofile(history)
            updates = 0.0
            for goal in times[1:]:
                t0 = time.perf_counter()
                s.advance(float(goal))
                s.synchronize()
                updates += time.perf_counter() - t0
                samples.append(sample())
                if history is not None:
                    host.tofile(history)
                with (output / "progress.jsonl").open("a") as f:
                    f.write(json.dumps({"budget": s.time, "steps": s.steps,
                                        "update_seconds": updates}) + "\n")
        finally:
            if history is not None:
                history.close()
        s.field(host)
        if not np.isfinite(host).all():
            raise RuntimeError("Non-finite field")
        arrival = s.arrival().ravel()
        np.savez_compressed(
            output / "labels.npz", indices=idx, states=states, times=times,
            values=np.stack(samples),
            arrival=arrival[idx] if weights is None else np.full(len(states), np.nan))
        if save_final:
            host.tofile(output / "final.f32")
        steps, max_dt = s.steps, s.dt_limit
    meta.update(
        status="complete", update_seconds=updates, steps=steps, max_internal_dt=max_dt,
        wall_seconds=time.perf_counter() - started, saved_final=bool(save_final),
        output_bytes=sum(x.stat().st_size for x in output.iterdir() if x.is_file()))
    (output / "meta.json").write_text(json.dumps(meta, indent=2))
    return meta
