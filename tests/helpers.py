"""Shared fixtures: physics configurations and golden-vector loaders."""

from pathlib import Path

import numpy as np

from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
from pursuit_evasion_b200.reversible.model import ReversibleConfig, VehicleLimits

GOLDEN = Path(__file__).resolve().parent / "golden"

# configs/reversible_free_a3.json of the reference (both accelerations 3 m/s^2)
A3 = ReversibleConfig(
    name="reversible_free_a3",
    pursuer=VehicleLimits(-1.0, 2.0, 3.0, 1.0),
    evader=VehicleLimits(-0.5, 1.0, 3.0, 2.0),
)
DEFAULT = ReversibleConfig()

# README smoke test of the reference: RelativeGrid(17, 12, 7, 7, 4.0), 0.2 s
CONFIG1_GRID = RelativeGrid(17, 12, 7, 7, 4.0)
# The 89M-cell table: 65 positions on [-8, 8], 48 headings, 21 x 21 speeds
CONFIG2_GRID = RelativeGrid(65, 48, 21, 21, 8.0)


def config_from_physics(physics, name="golden"):
    r, pmin, pmax, pa, pk, emin, emax, ea, ek = map(float, physics)
    return ReversibleConfig(name=name, pursuer=VehicleLimits(pmin, pmax, pa, pk),
                            evader=VehicleLimits(emin, emax, ea, ek),
                            capture_radius=r)


def relative_goldens():
    out = {}
    for path in sorted(GOLDEN.glob("relative5d_*.npz")):
        z = np.load(path)
        n, h, vp, ve = map(int, z["grid"])
        out[path.stem[len("relative5d_"):]] = dict(
            config=config_from_physics(z["physics"]),
            grid=RelativeGrid(n, h, vp, ve, float(z["extent"])),
            horizon=float(z["horizon"]), output_dt=float(z["output_dt"]),
            order=int(z["order"]), frames=z["frames"], arrival=z["arrival"],
            internal_steps=int(z["internal_steps"]),
            cfl_dt_limit=float(z["cfl_dt_limit"]),
        )
    return out


def world_goldens():
    out = {}
    for path in sorted(GOLDEN.glob("world8d_*.npz")):
        z = np.load(path)
        out[path.stem[len("world8d_"):]] = {k: z[k] for k in z.files}
    return out


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def square_goldens():
    """Golden vectors of the legacy 6D square game (tests/golden/square6d_*.npz,
    made by the reference executable native_square.cpp)."""
    return {p.stem[len("square6d_"):]: p for p in sorted(GOLDEN.glob("square6d_*.npz"))}
