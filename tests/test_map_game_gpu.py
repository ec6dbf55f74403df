"""gpu_map_game.solve on the device: the samples at node indices and at
continuous states are the saved frames at those nodes / interpolated with
the 256-corner stencil, the final field is the last frame, and the frames
are the WorldSolver map game's own (clearance floor, map surfaces)."""

import json

import numpy as np
import pytest

from pursuit_evasion_b200.reversible.gpu_map_game import interpolation_stencil, solve
from pursuit_evasion_b200.reversible.model import ReversibleConfig
from pursuit_evasion_b200.reversible.world_dp import WorldGrid, WorldSolver, output_times
from tests.helpers import bits
from tests.test_world_map_gpu import clearances

pytestmark = pytest.mark.gpu

MAP = ReversibleConfig(point_vehicles=False)


@pytest.mark.parametrize("fast", [False, True])
def test_map_game_solve_samples_and_frames(tmp_path, fast):
    grid = WorldGrid(9, 8, 5, 5, 3.0)
    pc, ec = clearances(grid)
    rng = np.random.default_rng(2)
    nodes = rng.integers(grid.states, size=50)
    meta = solve(MAP, grid, (pc, ec), tmp_path / "idx", horizon=0.2, output_dt=0.1,
                 query_indices=nodes, save_final=True, save_history=True, fast=fast)
    assert meta["status"] == "complete" and meta["schema"] == "footprint_map_game8d_v1"
    times = output_times(0.2, 0.1)
    frames = np.fromfile(tmp_path / "idx" / "fields.f32", np.float32).reshape(len(times), -1)
    labels = np.load(tmp_path / "idx" / "labels.npz")
    np.testing.assert_array_equal(labels["values"], frames[:, nodes])
    np.testing.assert_array_equal(np.fromfile(tmp_path / "idx" / "final.f32", np.float32),
                                  frames[-1])
    with WorldSolver(MAP, grid, cfl=0.7, avoid="clearance", fast=fast) as s:
        s.set_clearance(pc, ec)
        s.init_map()
        np.testing.assert_array_equal(bits(s.field().ravel()), bits(frames[0]))
        for goal in times[1:]:  # the solve's frame boundaries
            s.advance(float(goal))
        np.testing.assert_array_equal(bits(s.field().ravel()), bits(frames[-1]))
        assert meta["steps"] == s.steps
    # continuous states
    axes = grid.axes(MAP)
    lo = np.array([a[0] for a in axes])
    hi = np.array([a[-1] for a in axes])
    states = lo + (hi - lo) * rng.random((30, 8))
    solve(MAP, grid, (pc, ec), tmp_path / "st", horizon=0.2, output_dt=0.1,
          query_states=states, fast=fast)
    values = np.load(tmp_path / "st" / "labels.npz")["values"]
    idx, w, _ = interpolation_stencil(states, axes, (2, 6))
    np.testing.assert_allclose(values, (frames[:, idx] * w).sum(-1), rtol=1e-6, atol=1e-6)
    assert json.loads((tmp_path / "st" / "meta.json").read_text())["query_count"] == 30
