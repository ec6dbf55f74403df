"""Host-side checks of the compact contact solve driver: option errors
before any device work, and the sign-preserving float16 history."""

import numpy as np
import pytest

from pursuit_evasion_b200.local_game import reference
from pursuit_evasion_b200.local_game.geometry import CircleArena
from pursuit_evasion_b200.reversible.model import ReversibleConfig, VehicleLimits

CONFIG = ReversibleConfig(
    name="contact_a3", pursuer=VehicleLimits(-1.0, 2.0, 3.0, 1.0),
    evader=VehicleLimits(-0.5, 1.0, 3.0, 2.0), boundary_rule="collision_constrained",
    point_vehicles=False, capture_rule="rectangle_contact")
ARENA = CircleArena([[0.4, 0.3, 0.3]], 1.5)
OPTIONS = dict(headings=8, position_step=0.5, horizon=0.3, output_dt=0.1, exit_radius=1.5,
               retain_history=True, frames=3, per_frame=8, seed=5, log=None)


def test_solve_rejects_point_vehicle_rules(tmp_path):
    with pytest.raises(ValueError, match="finite-body"):
        reference.solve(ReversibleConfig(), ARENA, tmp_path / "x", **OPTIONS)
    with pytest.raises(ValueError, match="integer control periods"):
        reference.solve(CONFIG, ARENA, tmp_path / "y", **{**OPTIONS, "output_dt": 0.07})


def test_half_precision_history_keeps_the_sign(tmp_path):
    values = np.array([1e-9, -1e-9, 0.0, 0.5, -2.0], np.float32)
    with (tmp_path / "h.f16").open("wb") as f:
        reference.write_half_preserving_sign(values, f)
    back = np.fromfile(tmp_path / "h.f16", np.float16)
    assert back[0] > 0 and back[1] < 0 and back[2] == 0
    np.testing.assert_array_equal(back[3:], np.float16([0.5, -2.0]))


def test_first_crossing_interpolates_the_frame_before():
    times = [0.0, 0.1, 0.2]
    values = np.array([[1.0, -1.0, 2.0, np.nan], [0.5, -2.0, 1.0, 1.0], [-0.5, -3.0, 0.5, -1.0]])
    t = reference.first_crossing(times, values)
    np.testing.assert_allclose(t[:3], [0.15, 0.0, np.nan], equal_nan=True)
    assert t[3] == pytest.approx(0.15)
