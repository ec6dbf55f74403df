"""The reference GPU solve's extra keywords on the device
(gpu_relative.py:67-101, :156-226, :298-307): rectangle-contact capture
blocks, the local exit and probes.  The check is the oracle stage
(oracle/relative5d.c) with the exit restated around it: cells with
x^2 + y^2 > R^2 hold R and never arrive; every other cell updates as
without an exit, reading R from its exited neighbours.  The exit decision
is made in the arithmetic of the precision's kernel: double for float64
local arithmetic, float32 without contraction for float32."""

import json

import numpy as np
import pytest

from pursuit_evasion_b200.local_game.geometry import Footprint
from pursuit_evasion_b200.reversible.free_dp import (
    RelativeGrid,
    capture_plane,
    output_times,
    probe_stencils,
    solve,
)
from pursuit_evasion_b200.reversible.model import ReversibleConfig, VehicleLimits
from pursuit_evasion_b200.reversible.relative_solver import RelativeSolver
from tests.helpers import A3, bits
from tests.test_relative_gpu import assert_fast_close

pytestmark = pytest.mark.gpu

BODIES = (Footprint(0.8, 0.5), Footprint(0.4, 0.25))
CONTACT = ReversibleConfig(
    pursuer=VehicleLimits(-1.0, 2.0, 3.0, 1.0), evader=VehicleLimits(-0.5, 1.0, 3.0, 2.0),
    point_vehicles=False, capture_rule="rectangle_contact")
GRID = RelativeGrid(21, 12, 5, 5, 3.0)


def exit_mask(grid, radius, precision):
    """x^2 + y^2 > R^2 per (y, x) cell, as the reference kernel of that
    precision evaluates it with its 10-digit literal."""
    r2 = float(f"{radius ** 2:.9e}")
    n = grid.positions
    if precision == "float64":
        dx = 2 * grid.extent / (n - 1)
        c = -grid.extent + np.arange(n) * dx
        return c[None, :] * c[None, :] + c[:, None] * c[:, None] > r2
    w = np.float32(grid.extent)
    dx = np.float32(2) * w / np.float32(n - 1)
    c = -w + np.arange(n, dtype=np.float32) * dx
    return (c[None, :] * c[None, :] + c[:, None] * c[:, None]) > np.float32(r2)


def oracle_frames(oracle, config, grid, initial, radius, times, order, precision):
    """Frames and arrival of the oracle solve with the exit restated."""
    cfg = oracle.rel_cfg(config, grid, order=order)
    limit = oracle.rel_cfl_limit(cfg)
    r = np.float32(float(f"{radius:.9e}")) if radius else None
    mask = (np.broadcast_to(exit_mask(grid, radius, precision), grid.shape).ravel()
            if radius else None)
    a = np.ascontiguousarray(initial, np.float32).ravel().copy()
    b = np.empty_like(a)
    arrival = np.where(a <= 0, np.float32(0), np.float32(np.nan)).astype(np.float32)

    def hold(v):
        if mask is not None:
            v[mask] = r
            arrival[mask] = np.nan

    frames, t = [a.copy()], 0.0
    for goal in times[1:]:
        while t < goal - 1e-12:
            dt = min(limit, goal - t)
            rc, _ = oracle.rel_stage_f32(cfg, a, b, arrival, dt, t, 0)
            assert rc == 0
            hold(b)
            if order == 2:
                rc, _ = oracle.rel_stage_f32(cfg, b, a, arrival, dt, t, 1)
                assert rc == 0
                hold(a)
            else:
                a, b = b, a
            t += dt
        frames.append(a.copy())
    return np.array(frames), arrival


def gpu_frames(config, grid, plane, radius, times, order, precision):
    with RelativeSolver(config, grid, order=order, local_precision=precision) as s:
        s.set_exit(radius)
        s.initialize_plane(plane)
        frames = [s.field().ravel().copy()]
        for goal in times[1:]:
            s.advance(goal)
            frames.append(s.field().ravel().copy())
        return np.array(frames), s.arrival().ravel().copy()


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("contact, radius", [(False, 2.2), (True, None), (True, 2.6)],
                         ids=["exit", "contact", "contact-exit"])
def test_exact_path_with_keywords_matches_oracle_bitwise(oracle, order, contact, radius):
    config = CONTACT if contact else A3
    plane = capture_plane(config, GRID, BODIES if contact else None, radius)
    times = output_times(0.3, 0.1)
    ref, ref_arrival = oracle_frames(oracle, config, GRID, np.broadcast_to(plane, GRID.shape),
                                     radius, times, order, "float64")
    got, arrival = gpu_frames(config, GRID, plane, radius, times, order, "float64")
    np.testing.assert_array_equal(bits(got), bits(ref))
    np.testing.assert_array_equal(bits(arrival), bits(ref_arrival))
    if radius:
        mask = np.broadcast_to(exit_mask(GRID, radius, "float64"), GRID.shape).ravel()
        assert np.all(got[-1][mask] == np.float32(radius))
        assert np.all(np.isnan(arrival[mask]))


@pytest.mark.parametrize("contact, radius", [(False, 2.2), (True, 2.6)])
def test_fast_path_with_keywords_matches_oracle(oracle, contact, radius):
    config = CONTACT if contact else A3
    plane = capture_plane(config, GRID, BODIES if contact else None, radius)
    times = output_times(0.3, 0.1)
    ref, _ = oracle_frames(oracle, config, GRID, np.broadcast_to(plane, GRID.shape), radius,
                           times, 2, "float32")
    got, _ = gpu_frames(config, GRID, plane, radius, times, 2, "float32")
    assert_fast_close(got, ref)
    mask = np.broadcast_to(exit_mask(GRID, radius, "float32"), GRID.shape).ravel()
    assert np.all(got[-1][mask] == np.float32(radius))


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_solve_writes_probes_and_keyword_meta(tmp_path, precision):
    rng = np.random.default_rng(11)
    n = 40
    states = np.column_stack([
        rng.uniform(-3, 3, n), rng.uniform(-3, 3, n), rng.uniform(-4, 4, n),
        rng.uniform(-1, 2, n), rng.uniform(-0.5, 1, n)])
    meta = solve(CONTACT, GRID, tmp_path / "t", horizon=0.3, output_dt=0.1,
                 local_precision=precision, capture_footprints=BODIES, exit_radius=2.6,
                 probes=states)
    assert meta["capture_rule"] == "rectangle_contact"
    assert meta["local_exit_radius"] == 2.6
    assert meta["capture_footprints"]["pursuer"] == {"length": 0.8, "width": 0.5}
    assert np.array_equal(np.array(meta["probe_states"]), states)
    saved = json.loads((tmp_path / "t" / "meta.json").read_text())
    assert saved["status"] == "complete" and saved["probe_states"] is not None
    frames = np.fromfile(tmp_path / "t" / "fields.f32", np.float32).reshape(4, -1)
    probes = np.fromfile(tmp_path / "t" / "probes.f64", np.float64).reshape(4, n)
    _, idx, w = probe_stencils(CONTACT, GRID, states)
    want = (frames[:, idx].astype(np.float64) * w).sum(-1)
    np.testing.assert_allclose(probes, want, rtol=1e-12, atol=1e-12)
    # the frames are the keyword solve itself
    got, _ = gpu_frames(CONTACT, GRID, capture_plane(CONTACT, GRID, BODIES, 2.6), 2.6,
                        output_times(0.3, 0.1), 2, precision)
    np.testing.assert_array_equal(bits(frames), bits(got))


def test_exit_clears_when_disabled():
    plane = capture_plane(A3, GRID, exit_radius=2.2)
    times = output_times(0.1, 0.1)
    with RelativeSolver(A3, GRID, local_precision="float64") as s:
        s.set_exit(2.2)
        s.set_exit(None)
        s.initialize_plane(plane)
        s.advance(0.1)
        field = s.field().ravel()
    with RelativeSolver(A3, GRID, local_precision="float64") as s:
        s.initialize_plane(plane)
        s.advance(0.1)
        np.testing.assert_array_equal(bits(field), bits(s.field().ravel()))
    assert len(times) == 2
