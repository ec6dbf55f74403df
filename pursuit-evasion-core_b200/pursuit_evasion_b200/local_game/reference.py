"""Streaming solves of the compact contact game and queries of their signed
history.

The interface is the reference's local_game/reference.py: `solve` (:138-369)
builds both vehicle grids and the pair domain, samples observation /
query groups, and runs the packed min-max backup for `horizon /
control_dt` steps, saving at every `output_dt` the query labels, an atomic
float32 checkpoint (for `resume`) and, with `retain_history`, the signed
field as sign-preserving float16; `ContactReference` (:370-454) reads a
completed folder back (stencils over the pair domain, fields by budget, and
the first zero crossing as the capture time).  Folder layout and metadata
keys are the reference's, so folders interoperate.

Here the backups run in the fused one-launch kernel of csrc/capi_compact.cu
with the field resident on the device (pe_compact_*), the grids are built by
the GPU geometry of local_game/engine.py, and the labels come from the
device query of the packed field.
"""

from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path
import shutil
import time

import numpy as np

from ..reversible.model import ReversibleConfig
from .engine import GeometryEngine
from .geometry import CircleArena
from .grid_game import (
    PairDomain,
    VehicleGrid,
    backup_packed,
    initialize_packed,
    make_grid,
    packed_gpu_arrays,
)

_CHUNK = 2_000_000


def write_half_preserving_sign(values, file):
    """Append `values` as float16, keeping the sign of values that round to
    zero (the history's zero-sublevel convention needs the sign)."""
    tiny = np.nextafter(np.float16(0), np.float16(1))
    for start in range(0, len(values), _CHUNK):
        x = np.asarray(values[start:start + _CHUNK])
        h = x.astype(np.float16)
        underflow = h == 0
        h[underflow & (x > 0)] = tiny
        h[underflow & (x < 0)] = -tiny
        h.tofile(file)


def _wrap(angle):
    return np.mod(np.asarray(angle) + np.pi, 2 * np.pi) - np.pi


def sample_queries(p, e, domain, arena, config, *, frames=192, per_frame=256, seed=1031):
    """Observation / query groups of the solve's labels (reference.py:20-119):
    per frame, a pursuer pose with at least 30 evader states inside the exit
    radius, `per_frame` pairs at that pose that are not in contact, and a
    jittered sensor pose that is clear; then half of the query states are
    moved off the grid (position, heading and speed jitter) where the moved
    pair stays legal, separated, inside the exit radius and supported by
    both grids."""
    rng = np.random.default_rng(seed)
    observation, p_ids, e_ids, frame_ids = [], [], [], []
    for f in range(frames):
        for _ in range(1000):
            i = int(rng.integers(len(p.states)))
            pose = p.states[i, :3].copy()
            near = np.flatnonzero(np.linalg.norm(e.states[:, :2] - pose[:2], axis=1)
                                  <= domain.exit_radius - 0.1)
            if len(near) < 30:
                continue
            j = rng.choice(near, per_frame * 3, replace=True)
            same_pose = np.flatnonzero(np.all(p.states[:, :3] == pose, axis=1))
            ii = rng.choice(same_pose, len(j), replace=True)
            pair = np.concatenate([p.states[ii], e.states[j]], 1)
            apart = arena.capture_value(pair) > 0.03
            ii, j = ii[apart][:per_frame], j[apart][:per_frame]
            if len(ii) < per_frame:
                continue
            sensor = pose.copy()
            for _ in range(20):
                sensor = pose + np.array([rng.uniform(-0.11, 0.11), rng.uniform(-0.11, 0.11),
                                          rng.uniform(-0.11, 0.11)])
                if arena.clearance(np.r_[sensor, 0], "pursuer") > 1e-4:
                    break
            else:
                sensor = pose.copy()
            observation.append([*sensor, 0])
            p_ids.extend(ii)
            e_ids.extend(j)
            frame_ids.extend([f] * per_frame)
            break
        else:
            raise ValueError("Could not sample a legal observation/query group")
    pi, ei = np.array(p_ids, np.int32), np.array(e_ids, np.int32)
    local = domain.lookup[domain.p_position[pi], ei]
    assert (local >= 0).all()
    compact = domain.offsets[pi] + local
    states = np.concatenate([p.states[pi], e.states[ei]], 1)
    proposal = states.copy()
    move = rng.random(len(states)) < 0.5
    for k, limits in ((0, config.pursuer), (4, config.evader)):
        proposal[:, k:k + 2] += rng.uniform(-0.12, 0.12, (len(states), 2))
        proposal[:, k + 2] = _wrap(proposal[:, k + 2] + rng.uniform(-0.15, 0.15, len(states)))
        proposal[:, k + 3] = np.clip(proposal[:, k + 3] + rng.uniform(-0.1, 0.1, len(states)),
                                     limits.speed_min, limits.speed_max)
    p_engine = GeometryEngine(arena, config.pursuer, "pursuer", control_dt=config.control_dt)
    e_engine = GeometryEngine(arena, config.evader, "evader", control_dt=config.control_dt)
    legal = p_engine.backup_safe(proposal[:, :4]) & e_engine.backup_safe(proposal[:, 4:])
    legal &= arena.capture_value(proposal) > 0.03
    legal &= np.linalg.norm(proposal[:, :2] - proposal[:, 4:6], axis=1) < \
        domain.exit_radius - 0.02
    legal &= p.stencil(proposal[:, :4])[2] & e.stencil(proposal[:, 4:])[2]
    move &= legal
    states[move] = proposal[move]
    return dict(frames=np.array(observation), frame_ids=np.array(frame_ids, np.int32),
                p_indices=pi, e_indices=ei, original_compact_indices=compact,
                states=states, continuous=move)


def _spec(config, arena, **options):
    spec = dict(config=config.to_dict(), arena=arena.to_dict(), query_version=3, **options)
    return spec, hashlib.sha256(json.dumps(spec, sort_keys=True).encode()).hexdigest()


def _atomic_json(path, value):
    tmp = path.with_suffix(".tmp")
    tmp.write_text(json.dumps(value, indent=2))
    os.replace(tmp, path)


def solve(config, arena, output, *, headings=16, position_step=0.3, horizon=2.0,
          output_dt=0.25, exit_radius=3.0, retain_history=False, frames=192, per_frame=256,
          seed=1031, max_gb=7.6, device=0, log=print):
    """Solve the finite-body contact game into `output`, resuming a folder
    of the same setup (returns its metadata at once if it is complete)."""
    if (config.capture_rule != "rectangle_contact"
            or config.boundary_rule != "collision_constrained" or config.point_vehicles):
        raise ValueError("Use the explicit finite-body collision-constrained contact game")
    output = Path(output)
    output.mkdir(parents=True, exist_ok=True)
    dt = config.control_dt
    steps, every = round(horizon / dt), round(output_dt / dt)
    if (min(steps, every) < 1 or not np.isclose(steps * dt, horizon)
            or not np.isclose(every * dt, output_dt)):
        raise ValueError("Budgets must be integer control periods")
    spec, signature = _spec(config, arena, headings=headings, position_step=position_step,
                            horizon=horizon, output_dt=output_dt, exit_radius=exit_radius,
                            retain_history=retain_history, frames=frames,
                            per_frame=per_frame, seed=seed)
    meta_path = output / "meta.json"
    started = time.perf_counter()
    resume = meta_path.exists()
    if resume:
        meta = json.loads(meta_path.read_text())
        if meta["signature"] != signature:
            raise ValueError("Existing output belongs to another model/setup")
        if meta["status"] == "complete":
            return meta
        p = VehicleGrid.load(output / "p_grid.npz")
        e = VehicleGrid.load(output / "e_grid.npz")
        domain = PairDomain.load(output / "domain.npz")
        queries = dict(np.load(output / "queries.npz"))
    else:
        grids = {}
        for role, limits in (("pursuer", config.pursuer), ("evader", config.evader)):
            grids[role] = make_grid(arena, limits, role, headings=headings,
                                    position_step=position_step,
                                    speeds=np.linspace(limits.speed_min, limits.speed_max, 7),
                                    dt=dt, device=device)
        p, e = grids["pursuer"], grids["evader"]
        domain = PairDomain.build(p, e, exit_radius)
        p.save(output / "p_grid.npz")
        e.save(output / "e_grid.npz")
        domain.save(output / "domain.npz")
        queries = sample_queries(p, e, domain, arena, config, frames=frames,
                                 per_frame=per_frame, seed=seed)
        np.savez_compressed(output / "queries.npz", **queries)
        meta = dict(
            schema="local_contact_compact8d_v1", status="running", signature=signature,
            spec=spec, p_states=len(p.states), e_states=len(e.states),
            pair_states=domain.states, unpruned_pair_states=len(p.states) * len(e.states),
            history_dtype="float16_sign_preserved", completed_step=0, completed_outputs=0,
            times=[], update_seconds=0.0,
            interpolation="multilinear, omit invalid single-vehicle vertices and renormalize",
            action_constraint="continuous obstacle-free command plus one collision-free "
                              "constant-curvature braking backup",
            objective="capture by budget before center separation exceeds local radius; "
                      "range exit is local failure, not a physical capture",
            numerical_game="finite-grid semi-Lagrangian minP maxE, exact factorization of "
                           "the product interpolation; no dimension reduction",
            backend="b200_cuda_fused_packed_backup")
        _atomic_json(meta_path, meta)
    p.bind_geometry(arena, config.pursuer, "pursuer", dt, device)
    e.bind_geometry(arena, config.evader, "evader", dt, device)
    # one retained history plus the old and new checkpoints must fit together
    outputs = len(range(0, steps + 1, every))
    expected = ((outputs * 2 if retain_history else 0) + 8) * domain.states
    already = sum(f.stat().st_size for f in output.iterdir() if f.is_file())
    if shutil.disk_usage(output).free < max(0, expected - already) + 8 * 10**9:
        raise OSError("Insufficient disk space for history/checkpoint transaction plus8GB "
                      "reserve")
    arrays = packed_gpu_arrays(p, e, domain, max_gb=max_gb, tiled_output=True, device=device)
    pi, pw, pvalid, _, _ = p.stencil(queries["states"][:, :4])
    ei, ew, evalid, _, _ = e.stencil(queries["states"][:, 4:])
    if not (pvalid & evalid).all():
        raise ValueError("Generated query has no numerical support")
    host = np.empty(domain.states, np.float32)
    checkpoint = output / meta.get("checkpoint", "missing")
    if resume and meta["completed_outputs"] and checkpoint.exists():
        initialize_packed(arrays, p, e, domain, arena)  # creates the field
        arrays.set_field(np.fromfile(checkpoint, np.float32, count=domain.states))
        prior = np.load(output / "labels.npz")
        labels = list(prior["values"][:meta["completed_outputs"]])
        times = list(prior["times"][:meta["completed_outputs"]])
        start = meta["completed_step"]
    else:
        initialize_packed(arrays, p, e, domain, arena)
        labels, times, start = [], [], 0
    history = output / "fields.f16"
    if retain_history:
        with history.open("ab" if history.exists() else "wb") as f:
            f.truncate(meta["completed_outputs"] * domain.states * 2)

    def save_output(step):
        arrays.field(host)
        labels.append(arena.capture_value(queries["states"]).astype(np.float32) if step == 0
                      else arrays.query(pi, pw, ei, ew))
        times.append(step * dt)
        if retain_history:
            with history.open("ab") as f:
                write_half_preserving_sign(host, f)
        np.savez_compressed(output / "labels.npz", times=np.array(times),
                            values=np.stack(labels))
        name = f"checkpoint_{step:04d}.f32"
        partial = output / (name + ".partial")
        host.tofile(partial)
        os.replace(partial, output / name)
        old = meta.get("checkpoint")
        meta.update(completed_step=step, completed_outputs=len(times), times=times,
                    checkpoint=name, gpu_working_bytes=arrays["memory_bytes"],
                    host_working_bytes=domain.states * 4)
        _atomic_json(meta_path, meta)
        if old and old != name and (output / old).exists():
            (output / old).unlink()
        if log:
            log(f"budget {step * dt:.2f}s; states {domain.states:,}; "
                f"updates {meta['update_seconds']:.1f}s")

    try:
        if not labels:
            save_output(0)
        for step in range(start + 1, steps + 1):
            t0 = time.perf_counter()
            backup_packed(arrays, p, e, domain)
            arrays.synchronize()
            meta["update_seconds"] += time.perf_counter() - t0
            if step % every == 0 or step == steps:
                save_output(step)
    finally:
        arrays.close()
    meta.update(status="complete", wall_seconds_this_process=time.perf_counter() - started)
    (output / meta["checkpoint"]).unlink()
    meta.pop("checkpoint")
    meta["saved_bytes"] = sum(f.stat().st_size for f in output.iterdir()
                              if f.is_file() and f.name != "meta.json")
    _atomic_json(meta_path, meta)
    return meta


def first_crossing(times, values, valid=None):
    """Per query (columns of values [budget, query]), the budget at which the
    signed value first reaches zero, interpolated linearly from the frame
    before (reversible/map_game_field.py:83-98); NaN where it never does."""
    times = np.asarray(times, float)
    values = np.asarray(values, float)
    if values.ndim != 2 or len(times) != len(values) or np.any(np.diff(times) <= 0):
        raise ValueError("Expected increasing budgets and fields[budget,query]")
    hit = np.isfinite(values) & (values <= 0)
    found = hit.any(axis=0)
    first = hit.argmax(axis=0)
    prev = np.maximum(first - 1, 0)
    col = np.arange(values.shape[1])
    a, b = values[prev, col], values[first, col]
    frac = np.divide(a, a - b, out=np.zeros_like(a), where=np.abs(a - b) > 1e-12)
    when = times[prev] + np.clip(frac, 0, 1) * (times[first] - times[prev])
    if valid is not None:
        found &= np.asarray(valid, bool)
    return np.where(found, when, np.nan)


class ContactReference:
    """A completed solve with its signed history, read back for queries of
    8D states [xP, yP, thP, vP, xE, yE, thE, vE]."""

    def __init__(self, folder, device=0):
        self.folder = Path(folder)
        self.meta = json.loads((self.folder / "meta.json").read_text())
        if self.meta["status"] != "complete" or not self.meta["spec"]["retain_history"]:
            raise ValueError("A complete signed history is required")
        if not (self.folder / "fields.f16").exists():
            raise ValueError("History was not retained; regenerate into a new output folder")
        spec = self.meta["spec"]
        self.config = ReversibleConfig.from_dict(spec["config"])
        self.arena = CircleArena.from_dict(spec["arena"])
        self.p = VehicleGrid.load(self.folder / "p_grid.npz")
        self.e = VehicleGrid.load(self.folder / "e_grid.npz")
        self.domain = PairDomain.load(self.folder / "domain.npz")
        dt = self.config.control_dt
        self.p.bind_geometry(self.arena, self.config.pursuer, "pursuer", dt, device)
        self.e.bind_geometry(self.arena, self.config.evader, "evader", dt, device)
        self.times = np.array(self.meta["times"])
        self.horizon = self.times[-1]
        path = self.folder / "fields.f16"
        if path.stat().st_size != len(self.times) * self.domain.states * 2:
            raise ValueError("Incomplete history length")
        self.values = np.memmap(path, np.float16, mode="r",
                                shape=(len(self.times), self.domain.states))

    def stencil(self, s):
        """Pair-domain ids and product weights [n, 16, 16], which product
        vertices are inside the domain, validity of both car stencils, and
        whether the centres are within the exit radius."""
        s = np.asarray(s, float)
        batch = s.shape[:-1]
        flat = s.reshape(-1, 8)
        pi, pw, pv, _, _ = self.p.stencil(flat[:, :4])
        ei, ew, ev, _, _ = self.e.stencil(flat[:, 4:])
        rank = self.domain.lookup[self.domain.p_position[pi][:, :, None], ei[:, None, :]]
        ids = self.domain.offsets[pi][:, :, None] + np.maximum(rank, 0)
        weights = pw[:, :, None] * ew[:, None, :]
        inside = np.linalg.norm(flat[:, :2] - flat[:, 4:6], axis=1) <= self.domain.exit_radius
        return ids, weights, rank >= 0, pv & ev, inside, batch

    def fields(self, s):
        """Signed value at every budget of the history, [budgets, n]."""
        ids, w, kept, valid, inside, batch = self.stencil(s)
        exit_value = self.domain.exit_radius
        vertex = np.where(kept[None], self.values[:, ids].astype(np.float32), exit_value)
        values = np.sum(vertex * w[None], axis=(-1, -2))
        contact = self.arena.capture_value(np.asarray(s).reshape(-1, 8))
        values = np.minimum(values, contact[None])
        values = np.where(inside[None], values, exit_value)
        values[:, ~valid] = np.nan
        values[0, valid & inside] = contact[valid & inside]
        return values, valid & inside, batch

    def field(self, s, budget=None):
        values, _, batch = self.fields(s)
        budget = self.horizon if budget is None else budget
        if not 0 <= budget <= self.horizon:
            raise ValueError("Budget outside reference")
        i = min(np.searchsorted(self.times, budget, side="right") - 1, len(self.times) - 2)
        f = (budget - self.times[i]) / (self.times[i + 1] - self.times[i])
        return ((1 - f) * values[i] + f * values[i + 1]).reshape(batch)

    def time_value(self, s):
        values, valid, batch = self.fields(s)
        return first_crossing(self.times, values, valid).reshape(batch)
