"""Golden vehicle grids of the compact contact game, written by the
reference's own make_grid (local_game/grid_game.py:158-196, with its OpenMP
geometry library local_game/native_geometry.cpp, which it compiles itself)
on a small arena with circular obstacles, for both cars; and the reference
stencil of random states against the bound evader grid, including states
without multilinear support, which take the nearest-supported fallback
(grid_game.py:38-79).  The GPU geometry and make_grid of this package are
checked against them (tests/test_vehicle_grid_gpu.py).

Run in a container where the reference tree is mounted:
    python tests/golden/make_vehicle_grid_golden.py
"""

import os
from pathlib import Path
import sys

import numpy as np

HERE = Path(__file__).resolve().parent
# the reference tree: PE_REFERENCE_ROOT, by default where it is mounted here
sys.path.insert(0, os.path.join(os.environ.get("PE_REFERENCE_ROOT", "/root/reference"), "src"))

from pursuit_evasion.local_game.geometry import CircleArena  # noqa: E402
from pursuit_evasion.local_game.grid_game import make_grid  # noqa: E402
from pursuit_evasion.reversible.model import VehicleLimits  # noqa: E402

# a 3 m square with two posts; the a3 limits (configs/reversible_free_a3.json)
CIRCLES = [[0.3, 0.2, 0.35], [-0.6, -0.4, 0.3]]
HALF_WIDTH = 1.5
STEP, HEADINGS, DT = 0.5, 8, 0.05
LIMITS = {"pursuer": (-1.0, 2.0, 3.0, 1.0), "evader": (-0.5, 1.0, 3.0, 2.0)}


def main():
    arena = CircleArena(CIRCLES, HALF_WIDTH)
    out = {"circles": np.array(CIRCLES), "half_width": HALF_WIDTH,
           "options": np.array([STEP, HEADINGS, DT])}
    grids = {}
    for role, lim in LIMITS.items():
        limits = VehicleLimits(*lim)
        g = make_grid(arena, limits, role, position_step=STEP, headings=HEADINGS, dt=DT)
        grids[role] = g
        out[f"{role}_limits"] = np.array(lim)
        for key in ("states", "dense_to_compact", "controls", "successors", "weights",
                    "allowed", "retained_mass"):
            out[f"{role}_{key}"] = getattr(g, key)
        print(role, len(g.states), "states,", int(g.allowed.sum()), "allowed actions")
    # random evader states, most of them close to the posts and the walls
    # at speed, where whole stencils can be illegal
    rng = np.random.default_rng(7)
    e = grids["evader"]
    n = 3000
    pts = rng.uniform(-HALF_WIDTH + 0.15, HALF_WIDTH - 0.15, (n, 2))
    m = 2 * n // 3
    near = rng.integers(len(CIRCLES), size=m)
    ang = rng.uniform(-np.pi, np.pi, m)
    rad = np.array(CIRCLES)[near, 2] + rng.uniform(0.12, 0.3, m)
    pts[:m] = np.array(CIRCLES)[near, :2] + rad[:, None] * np.c_[np.cos(ang), np.sin(ang)]
    speed = np.where(np.arange(n) < m, rng.uniform(0.6, 1.0, n), rng.uniform(-0.5, 1.0, n))
    q = np.c_[pts, rng.uniform(-np.pi, np.pi, n), speed]
    ids, w, valid, _, mass = e.stencil(q)
    out["query_states"] = q
    out["query_ids"], out["query_weights"], out["query_valid"] = ids, w, valid
    out["query_fallback"] = valid & (mass <= 1e-9)
    out["query_clearance"] = arena.clearance(q, "evader")
    out["query_backup_safe"] = e._engine.backup_safe(q)
    print("queries:", int(valid.sum()), "valid,", int(out["query_fallback"].sum()),
          "through the fallback")
    np.savez_compressed(HERE / "vehicle_grid_posts3m.npz", **out)


if __name__ == "__main__":
    main()
