"""The compact contact solve driver (local_game/reference.py) on a small
arena: grids from the GPU geometry, sampled queries, fused packed backups,
labels, float16 history and checkpoints.  A solve interrupted after a few
backups and resumed from its checkpoint writes the same history and labels
as an uninterrupted one, bit for bit; the folder reads back through
ContactReference (the budget-0 field is the contact value, labels equal
the history's field at the query states, capture times lie in the
horizon); and a completed folder is returned as it is."""

import numpy as np
import pytest

from pursuit_evasion_b200.local_game import grid_game, reference
from pursuit_evasion_b200.local_game.geometry import CircleArena
from pursuit_evasion_b200.reversible.model import ReversibleConfig, VehicleLimits

pytestmark = pytest.mark.gpu

CONFIG = ReversibleConfig(
    name="contact_a3", pursuer=VehicleLimits(-1.0, 2.0, 3.0, 1.0),
    evader=VehicleLimits(-0.5, 1.0, 3.0, 2.0), boundary_rule="collision_constrained",
    point_vehicles=False, capture_rule="rectangle_contact")
ARENA = CircleArena([[0.4, 0.3, 0.3]], 1.5)
OPTIONS = dict(headings=8, position_step=0.5, horizon=0.3, output_dt=0.1, exit_radius=1.5,
               retain_history=True, frames=3, per_frame=8, seed=5, log=None)


def test_resumed_solve_equals_uninterrupted_and_reads_back(tmp_path, monkeypatch):
    full = reference.solve(CONFIG, ARENA, tmp_path / "full", **OPTIONS)
    assert full["status"] == "complete" and full["completed_step"] == 6
    assert full["times"] == pytest.approx([0.0, 0.1, 0.2, 0.3])

    # interrupt after the third backup (one output saved past budget 0)
    calls = {"n": 0}
    real = reference.backup_packed

    def failing(*args):
        calls["n"] += 1
        if calls["n"] == 4:
            raise KeyboardInterrupt
        return real(*args)

    monkeypatch.setattr(reference, "backup_packed", failing)
    with pytest.raises(KeyboardInterrupt):
        reference.solve(CONFIG, ARENA, tmp_path / "resumed", **OPTIONS)
    monkeypatch.setattr(reference, "backup_packed", real)
    partial = reference.json.loads((tmp_path / "resumed" / "meta.json").read_text())
    assert partial["status"] == "running" and partial["completed_step"] == 2
    resumed = reference.solve(CONFIG, ARENA, tmp_path / "resumed", **OPTIONS)
    assert resumed["status"] == "complete"
    for name in ("fields.f16",):
        a = (tmp_path / "full" / name).read_bytes()
        b = (tmp_path / "resumed" / name).read_bytes()
        assert a == b
    la, lb = (np.load(tmp_path / d / "labels.npz") for d in ("full", "resumed"))
    np.testing.assert_array_equal(la["values"], lb["values"])
    # a completed folder is returned as it is
    again = reference.solve(CONFIG, ARENA, tmp_path / "full", **OPTIONS)
    assert again == full or again["status"] == "complete"

    ref = reference.ContactReference(tmp_path / "full")
    q = dict(np.load(tmp_path / "full" / "queries.npz"))
    states = q["states"]
    values, valid, _ = ref.fields(states)
    assert valid.all()
    np.testing.assert_allclose(values[0], ARENA.capture_value(states), rtol=0, atol=1e-12)
    # labels are the float32 field at the queries; the reader also takes the
    # contact value at the state as a bound, and its history is float16
    contact = ARENA.capture_value(states)
    np.testing.assert_allclose(values[1:], np.minimum(la["values"][1:], contact), rtol=0,
                               atol=2e-3)
    t = ref.time_value(states)
    assert np.all(np.isnan(t) | ((t >= 0) & (t <= 0.3 + 1e-12)))
    assert ref.field(states, 0.05).shape == (len(states),)
    # the history never rises: capture by a budget stays capture later
    assert np.all(np.diff(values, axis=0) <= 1e-3)


def test_make_grid_keeps_states_with_an_action():
    g = grid_game.make_grid(ARENA, CONFIG.evader, "evader", position_step=0.5, headings=8)
    assert g.allowed.any(axis=1).all()
    assert (g.dense_to_compact >= 0).sum() == len(g.states)
