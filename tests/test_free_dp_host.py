"""Host logic of the drop-in free_dp API (no GPU work): grid and option
validation, frame times, the physics signature, and the guards that must
fail before anything is allocated or created (free_dp.py:145-176)."""

import json
from dataclasses import replace

import numpy as np
import pytest

from pursuit_evasion_b200.reversible.free_dp import (
    RelativeGrid,
    output_times,
    physics_signature,
    solve,
)
from pursuit_evasion_b200.reversible.model import ReversibleConfig
from tests.helpers import A3


def test_grid_shape_axes_and_validation():
    g = RelativeGrid(17, 12, 7, 7, 4.0)
    assert g.shape == (7, 7, 12, 17, 17) and g.states == 169932
    axes = g.axes(A3)
    assert axes[2][0] == -np.pi and len(axes[2]) == 12
    np.testing.assert_allclose(np.diff(axes[2]), 2 * np.pi / 12)
    assert axes[3][0] == -4 and axes[3][-1] == 4
    for bad in [dict(positions=2), dict(headings=3), dict(p_speeds=2),
                dict(e_speeds=1.5), dict(extent=0.0), dict(positions=True)]:
        with pytest.raises(ValueError):
            RelativeGrid(**{**g.to_dict(), **bad})


def test_output_times_match_reference_convention():
    np.testing.assert_allclose(output_times(0.2, 0.1), [0, 0.1, 0.2])
    np.testing.assert_allclose(output_times(0.25, 0.1), [0, 0.1, 0.2, 0.25])
    assert len(output_times(3.0, 0.1)) == 31


def test_physics_signature_ignores_map_placement():
    sig = physics_signature(A3)
    assert sig == physics_signature(replace(A3, arena_half_width=10))
    assert sig != physics_signature(replace(A3, capture_radius=0.4))
    assert set(sig) == {"capture_radius", "pursuer", "evader"}


def test_config_json_round_trip():
    text = json.dumps(A3.to_dict())
    assert ReversibleConfig.from_dict(json.loads(text)) == A3


def test_memory_guard_before_allocation(tmp_path):
    with pytest.raises(MemoryError):
        solve(ReversibleConfig(), RelativeGrid(101, 48, 13, 13, 4),
              tmp_path / "large", max_working_gb=0.001)
    assert not (tmp_path / "large").exists()


def test_invalid_options_and_existing_output(tmp_path):
    g = RelativeGrid(9, 8, 7, 7, 1.0)
    with pytest.raises(ValueError):
        solve(A3, g, tmp_path / "a", horizon=-1)
    with pytest.raises(ValueError):
        solve(A3, g, tmp_path / "a", cfl=1.5)
    with pytest.raises(ValueError):
        solve(A3, g, tmp_path / "a", order=3)
    with pytest.raises(ValueError):
        solve(A3, RelativeGrid(9, 8, 7, 7, 0.2), tmp_path / "a")
    with pytest.raises(ValueError):
        solve(A3, g, tmp_path / "a", tol=-1)
    rect = replace(A3, capture_rule="rectangle_contact", point_vehicles=False,
                   boundary_rule="collision_constrained")
    with pytest.raises(ValueError):
        solve(rect, g, tmp_path / "a")
    (tmp_path / "busy").mkdir()
    (tmp_path / "busy" / "x").write_text("keep")
    with pytest.raises(FileExistsError):
        solve(A3, g, tmp_path / "busy")
    assert (tmp_path / "busy" / "x").read_text() == "keep"
