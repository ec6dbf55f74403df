"""Golden relative successors from the REFERENCE Python model.

Imports pursuit-evasion-core's own model (src/pursuit_evasion/reversible/
model.py: joint_step, relative_state) and action catalogue
(controllers.py: action_catalogue) from the mounted reference tree, and
stores, for seeded random relative states and every one of the 9x9
pursuer x evader actions, the successor relative state after a held step:
    relative_state(joint_step([0,0,0,vP, x,y,psi,vE], u, w, dt))
Also stores known answers of integrated_speed.

Run where the reference is mounted:  python tests/golden/make_successor_golden.py
"""

import os
from pathlib import Path
import sys

import numpy as np

HERE = Path(__file__).resolve().parent
# the reference tree: PE_REFERENCE_ROOT, by default where it is mounted here
sys.path.insert(0, os.path.join(os.environ.get("PE_REFERENCE_ROOT", "/root/reference"), "src"))

from pursuit_evasion.reversible.model import (  # noqa: E402
    ReversibleConfig,
    VehicleLimits,
    integrated_speed,
    joint_step,
    relative_state,
)
from pursuit_evasion.reversible.controllers import action_catalogue  # noqa: E402


def main():
    config = ReversibleConfig(
        name="reversible_free_a3",
        pursuer=VehicleLimits(-1.0, 2.0, 3.0, 1.0),
        evader=VehicleLimits(-0.5, 1.0, 3.0, 2.0),
    )
    rng = np.random.default_rng(2024)
    n = 64
    rel = np.column_stack([
        rng.uniform(-4, 4, n), rng.uniform(-4, 4, n), rng.uniform(-np.pi, np.pi, n),
        rng.uniform(-1, 2, n), rng.uniform(-0.5, 1, n)])
    # include speeds at the bounds, where acceleration saturates
    rel[:4, 3] = [-1, 2, -1, 2]
    rel[4:8, 4] = [-0.5, 1, 1, -0.5]
    dts = np.array([0.01316, 0.05, 0.3])
    P = action_catalogue(config.pursuer)
    E = action_catalogue(config.evader)
    out = np.zeros((len(dts), n, 9, 9, 5))
    for t, dt in enumerate(dts):
        world = np.zeros((n, 8))
        world[:, 3] = rel[:, 3]
        world[:, 4] = rel[:, 0]
        world[:, 5] = rel[:, 1]
        world[:, 6] = rel[:, 2]
        world[:, 7] = rel[:, 4]
        nxt = joint_step(world[:, None, None, :], P[None, :, None, :],
                         E[None, None, :, :], dt, config)
        out[t] = relative_state(nxt)
    speeds = np.array([[1.5, 2.0, 1.0], [1.0, -2.0, 1.0], [1.0, -2.0, 0.5],
                       [-0.9, -3.0, 0.05], [0.0, 0.0, 0.3]])
    ans = np.array([integrated_speed(v, a, d, config.pursuer) for v, a, d in speeds])
    np.savez_compressed(HERE / "sl_successors.npz", states=rel, dts=dts,
                        successors=out, pursuer_actions=P, evader_actions=E,
                        speed_cases=speeds, speed_answers=ans)
    print("saved", out.shape)


if __name__ == "__main__":
    main()
