"""Vehicle grids of the compact contact game built by this package's GPU
geometry (csrc/vehicle_geometry_exact.cu) against the reference's own
make_grid on the same arena (golden vectors written by
tests/golden/make_vehicle_grid_golden.py): kept states, dense-to-compact
map, controls, allowed actions and successor stencils; and the stencil of
random states of the bound grid, including the nearest-supported fallback
for states whose multilinear corners are all illegal."""

from pathlib import Path

import numpy as np
import pytest

from pursuit_evasion_b200.local_game.engine import GeometryEngine
from pursuit_evasion_b200.local_game.geometry import CircleArena
from pursuit_evasion_b200.local_game.grid_game import make_grid
from pursuit_evasion_b200.reversible.model import VehicleLimits

pytestmark = pytest.mark.gpu

GOLDEN = np.load(Path(__file__).resolve().parent / "golden" / "vehicle_grid_posts3m.npz")


def arena():
    return CircleArena(GOLDEN["circles"], float(GOLDEN["half_width"]))


def build(role):
    step, headings, dt = GOLDEN["options"]
    return make_grid(arena(), VehicleLimits(*GOLDEN[f"{role}_limits"]), role,
                     position_step=float(step), headings=int(headings), dt=float(dt))


@pytest.mark.parametrize("role", ["pursuer", "evader"])
def test_make_grid_equals_the_reference_grid(role):
    g = build(role)
    for key in ("states", "dense_to_compact", "controls", "allowed", "successors"):
        np.testing.assert_array_equal(getattr(g, key), GOLDEN[f"{role}_{key}"], err_msg=key)
    np.testing.assert_allclose(g.weights, GOLDEN[f"{role}_weights"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(g.retained_mass, GOLDEN[f"{role}_retained_mass"], rtol=0,
                               atol=1e-9)


def test_geometry_queries_and_fallback_stencils_equal_the_reference():
    g = build("evader")
    q = GOLDEN["query_states"]
    engine = GeometryEngine(arena(), VehicleLimits(*GOLDEN["evader_limits"]), "evader",
                            control_dt=float(GOLDEN["options"][2]))
    np.testing.assert_allclose(engine.clearance(q), GOLDEN["query_clearance"], rtol=0,
                               atol=1e-12)
    np.testing.assert_array_equal(engine.backup_safe(q), GOLDEN["query_backup_safe"])
    ids, w, valid, _, _ = g.stencil(q)
    np.testing.assert_array_equal(valid, GOLDEN["query_valid"])
    np.testing.assert_array_equal(ids[valid], GOLDEN["query_ids"][valid])
    np.testing.assert_allclose(w[valid], GOLDEN["query_weights"][valid], rtol=0, atol=1e-6)
    assert GOLDEN["query_fallback"].sum() >= 10  # the fallback is exercised
