"""The obstacle map game on the 8D grid (gpu_map_game.py:45-50, :64-66):
each car's clearance per (x, y, heading) pose floors the pursuer's updates
(avoid mode 2) and limits the evader's initial value.  Exact stage against
the oracle restatement bit for bit from the same initial field; the initial
field itself against the oracle to within hypotf's last bit (device and host
libraries); the fast stage against the exact one."""

import numpy as np
import pytest

from pursuit_evasion_b200.reversible.world_dp import WorldGrid, WorldSolver
from tests import oracle_lib
from tests.helpers import A3, bits

pytestmark = pytest.mark.gpu


def clearances(grid):
    """Synthetic clearances: distance to a disc obstacle minus a heading-
    dependent body half-length (a stand-in for FootprintMap.clearance)."""
    x = np.linspace(-grid.extent, grid.extent, grid.positions)
    h = -np.pi + np.arange(grid.headings) * 2 * np.pi / grid.headings
    X, Y, H = np.meshgrid(x, x, h, indexing="ij")
    p = np.hypot(X - 0.7, Y + 0.4) - 0.6 - 0.15 * np.abs(np.cos(H))
    e = np.hypot(X + 0.5, Y - 0.9) - 0.5 - 0.1 * np.abs(np.sin(H))
    return p.astype(np.float32), e.astype(np.float32)


def cfg_of(grid, order):
    p, e = A3.pursuer, A3.evader
    return oracle_lib.W8Cfg(grid.positions, grid.headings, grid.p_speeds, grid.e_speeds,
                            order, 1, 0, grid.extent, A3.arena_half_width, A3.capture_radius,
                            p.speed_min, p.speed_max, e.speed_min, e.speed_max,
                            p.acceleration, e.acceleration, p.max_curvature,
                            e.max_curvature, 0.8)


@pytest.mark.parametrize("order", [1, 2])
def test_map_game_exact_stage_matches_oracle(oracle, order):
    grid = WorldGrid(7, 6, 4, 3, 3.0)
    pc, ec = clearances(grid)
    cfg = cfg_of(grid, order)
    ref0, ref_arr0 = oracle.w8_init_map(cfg, pc, ec)
    with WorldSolver(A3, grid, order=order, avoid="clearance") as s:
        s.set_clearance(pc, ec)
        s.init_map()
        first = s.field().ravel().copy()
        np.testing.assert_allclose(first, ref0, rtol=1e-6, atol=1e-6)
        assert (first <= 0).any() and (first > 0).any()
        # continue both from the device's initial field
        s.init_field(first)
        a, arrival = first.copy(), np.where(first <= 0, 0, np.nan).astype(np.float32)
        b = np.zeros_like(a)
        tau = 0.0
        for _ in range(6):
            dt = float(s.dt_limit)
            s.step(s.dt_limit)
            if order == 1:
                assert oracle.w8_stage_clear(cfg, a, b, None, arrival, dt, tau, pc) == 0
                a, b = b, a
            else:
                assert oracle.w8_stage_clear(cfg, a, b, None, arrival, dt, tau, pc) == 0
                assert oracle.w8_stage_clear(cfg, b, a, a, arrival, dt, tau, pc) == 0
            tau += s.dt_limit
        got = s.field().ravel()
        np.testing.assert_array_equal(bits(got), bits(a))
        np.testing.assert_array_equal(bits(s.arrival().ravel()), bits(arrival))
    # the floor holds: no value below -p_clear + 1e-6 of its pursuer pose
    floor = np.broadcast_to((-pc + np.float32(1e-6))[:, :, :, None, None, None, None, None],
                            grid.shape).ravel()
    assert np.all(got >= floor)


def test_map_game_fast_stage_tracks_exact():
    grid = WorldGrid(11, 9, 7, 7, 3.0)
    pc, ec = clearances(grid)
    out = {}
    for fast in (False, True):
        with WorldSolver(A3, grid, avoid="clearance", fast=fast) as s:
            s.set_clearance(pc, ec)
            s.init_map()
            for _ in range(10):
                s.step(s.dt_limit)
            out[fast] = s.field().ravel().astype(np.float64)
    diff = np.abs(out[True] - out[False])
    assert diff.max() < 1e-2 and diff.mean() < 3e-6


def test_map_game_needs_clearance_first():
    grid = WorldGrid(7, 6, 4, 3, 3.0)
    with WorldSolver(A3, grid, avoid="clearance") as s:
        with pytest.raises(Exception):
            s.init_map()
        with pytest.raises(ValueError):
            s.set_clearance(np.zeros((7, 7, 5)), np.zeros((7, 7, 5)))
