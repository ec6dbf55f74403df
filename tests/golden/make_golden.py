"""Generate the golden vectors under tests/golden/ from the REFERENCE itself.

Runs the reference executables compiled from the reference sources
(oracle/_ref/, recipe: oracle/Makefile `make ref`) on small grids and stores
their outputs as compressed .npz fixtures:

    relative5d_<name>.npz   native_relative.cpp: every frame of fields.f32,
                            arrival.f32, internal_steps, cfl_dt_limit
    world8d_<name>.npz      native_world.cpp: final frame and arrival

Run in a container where the reference tree is mounted:
    make -C oracle ref && python tests/golden/make_golden.py
"""

import json
from pathlib import Path
import subprocess
import sys
import tempfile

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "pursuit-evasion-core_b200"))

from tests.oracle_lib import REF_WORLD, run_reference_relative  # noqa: E402
from pursuit_evasion_b200.reversible.free_dp import RelativeGrid  # noqa: E402
from pursuit_evasion_b200.reversible.model import (  # noqa: E402
    ReversibleConfig,
    VehicleLimits,
)

A3 = ReversibleConfig(
    name="reversible_free_a3",
    pursuer=VehicleLimits(-1.0, 2.0, 3.0, 1.0),
    evader=VehicleLimits(-0.5, 1.0, 3.0, 2.0),
)
DEFAULT = ReversibleConfig()

RELATIVE_CASES = {
    # name: (config, grid, horizon, output_dt, order)
    "a3_7x6x5x5_o2": (A3, RelativeGrid(7, 6, 5, 5, 1.0), 0.06, 0.02, 2),
    "a3_7x6x5x5_o1": (A3, RelativeGrid(7, 6, 5, 5, 1.0), 0.06, 0.02, 1),
    "default_5x4x3x3_o2": (DEFAULT, RelativeGrid(5, 4, 3, 3, 1.0), 0.05, 0.025, 2),
    "a3_9x8x4x3_ext2_o2": (A3, RelativeGrid(9, 8, 4, 3, 2.0), 0.3, 0.1, 2),
}

WORLD_CASES = {
    # name: (n, nh, np, ne, extent, horizon, output_dt, order, linear)
    "default_5x4x3x3_o2_linear": (5, 4, 3, 3, 3.5, 0.02, 0.01, 2, 1),
    "default_5x4x3x3_o1_legacy": (5, 4, 3, 3, 3.5, 0.02, 0.01, 1, 0),
}


def relative_golden():
    for name, (config, grid, horizon, output_dt, order) in RELATIVE_CASES.items():
        folder, timing = run_reference_relative(
            config, grid, horizon=horizon, output_dt=output_dt, order=order,
            threads=2)
        count = int(np.ceil(horizon / output_dt - 1e-10)) + 1
        frames = np.fromfile(folder / "fields.f32", np.float32).reshape(
            count, *grid.shape)
        arrival = np.fromfile(folder / "arrival.f32", np.float32).reshape(grid.shape)
        p, e = config.pursuer, config.evader
        np.savez_compressed(
            HERE / f"relative5d_{name}.npz",
            frames=frames, arrival=arrival,
            internal_steps=timing["internal_steps"],
            cfl_dt_limit=timing["cfl_dt_limit"],
            grid=np.array([grid.positions, grid.headings, grid.p_speeds,
                           grid.e_speeds]),
            extent=grid.extent, horizon=horizon, output_dt=output_dt,
            order=order,
            physics=np.array([config.capture_radius, p.speed_min, p.speed_max,
                              p.acceleration, p.max_curvature, e.speed_min,
                              e.speed_max, e.acceleration, e.max_curvature]),
        )
        print(name, frames.shape, timing["internal_steps"])


def world_golden():
    c = DEFAULT
    p, e = c.pursuer, c.evader
    for name, (n, nh, np_, ne, extent, horizon, odt, order, linear) in (
            WORLD_CASES.items()):
        out = Path(tempfile.mkdtemp(prefix="pe_w8_"))
        options = {
            "positions": n, "headings": nh, "p-speeds": np_, "e-speeds": ne,
            "extent": extent, "arena": c.arena_half_width,
            "radius": c.capture_radius, "p-min": p.speed_min,
            "p-max": p.speed_max, "e-min": e.speed_min, "e-max": e.speed_max,
            "p-accel": p.acceleration, "e-accel": e.acceleration,
            "p-curvature": p.max_curvature, "e-curvature": e.max_curvature,
            "horizon": horizon, "output-dt": odt, "order": order, "cfl": 0.8,
            "threads": 2, "history": 0, "linear-speed-boundary": linear,
            "output": str(out),
        }
        cmd = [str(REF_WORLD)] + [str(x) for k, v in options.items()
                                  for x in ("--" + k, v)]
        subprocess.run(cmd, check=True, capture_output=True)
        timing = json.loads((out / "native_timing.json").read_text())
        shape = (n, n, nh, np_, n, n, nh, ne)
        final = np.fromfile(out / "final.f32", np.float32).reshape(shape)
        arrival = np.fromfile(out / "arrival.f32", np.float32).reshape(shape)
        np.savez_compressed(
            HERE / f"world8d_{name}.npz", final=final, arrival=arrival,
            internal_steps=timing["internal_steps"],
            grid=np.array([n, nh, np_, ne]), extent=extent, horizon=horizon,
            output_dt=odt, order=order, linear=linear,
            arena=c.arena_half_width,
            physics=np.array([c.capture_radius, p.speed_min, p.speed_max,
                              p.acceleration, p.max_curvature, e.speed_min,
                              e.speed_max, e.acceleration, e.max_curvature]),
        )
        print(name, shape, timing["internal_steps"])


if __name__ == "__main__":
    relative_golden()
    world_golden()
