"""Generate the compact 8D semi-Lagrangian backup golden vectors from the
REFERENCE itself.

Imports, in place and read-only, the reference's own test helpers
`fake_grid` and `brute_backup` (tests/test_compact_dp.py:12-51, the joint
action enumeration of the factorized backup), `PairDomain.build`
(src/pursuit_evasion/local_game/grid_game.py:289-313) and
`rectangle_separation` / `CircleArena`
(src/pursuit_evasion/local_game/geometry.py:15-45), and stores, per case,
the two vehicle grids, the pair domain, the capture field clamped at the
exit radius and the fields after each of `backups` brute-force backups.

    compact8d_<name>.npz   p_/e_ states, successors, weights, allowed;
                           domain p_position, lookup, e_indices, counts,
                           offsets; exit_radius; footprints; frames [B+1, np, ne]

Run in a container where the reference tree is mounted:
    python tests/golden/make_compact_golden.py
"""

import importlib.util
import os
from pathlib import Path
import sys

import numpy as np

HERE = Path(__file__).resolve().parent
# the reference tree: PE_REFERENCE_ROOT, by default where it is mounted here
REFERENCE = Path(os.environ.get("PE_REFERENCE_ROOT", "/root/reference"))

# (name, seed, p states, p actions, e states, e actions, exit radius, backups)
CASES = [
    ("seed114_5x3_7x4", 114, 5, 3, 7, 4, 1.2, 2),   # test_compact_dp.py:54-79
    ("seed57_5x3_7x4", 57, 5, 3, 7, 4, 1.2, 2),     # test_compact_dp.py:82-119
    ("seed7_24x9_30x9", 7, 24, 9, 30, 9, 1.2, 3),
    ("seed11_40x9_33x9", 11, 40, 9, 33, 9, 0.9, 2),
]


def load_reference():
    sys.path.insert(0, str(REFERENCE / "src"))
    spec = importlib.util.spec_from_file_location(
        "ref_test_compact_dp", REFERENCE / "tests" / "test_compact_dp.py")
    tests = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(tests)
    from pursuit_evasion.local_game.geometry import CircleArena, rectangle_separation
    from pursuit_evasion.local_game.grid_game import PairDomain

    return tests, CircleArena, rectangle_separation, PairDomain


def main():
    tests, CircleArena, rectangle_separation, PairDomain = load_reference()
    arena = CircleArena([], 3)
    for name, seed, n_p, a_p, n_e, a_e, radius, backups in CASES:
        rng = np.random.default_rng(seed)
        p, e = tests.fake_grid(n_p, a_p, rng), tests.fake_grid(n_e, a_e, rng)
        domain = PairDomain.build(p, e, radius)
        field = rectangle_separation(p.states[:, None], e.states[None],
                                     arena.pursuer, arena.evader)
        far = np.linalg.norm(p.states[:, None, :2] - e.states[None, :, :2], axis=-1) > radius
        field = np.where(far, radius, field)
        frames = [field]
        for _ in range(backups):
            frames.append(tests.brute_backup(frames[-1], p, e, radius))
        np.savez_compressed(
            HERE / f"compact8d_{name}.npz",
            p_states=p.states, p_successors=p.successors, p_weights=p.weights,
            p_allowed=p.allowed,
            e_states=e.states, e_successors=e.successors, e_weights=e.weights,
            e_allowed=e.allowed,
            p_position=domain.p_position, lookup=domain.lookup,
            e_indices=domain.e_indices, counts=domain.counts, offsets=domain.offsets,
            exit_radius=radius,
            footprints=np.array([arena.pursuer.length, arena.pursuer.width,
                                 arena.evader.length, arena.evader.width]),
            frames=np.array(frames),
        )
        print(name, "frames", np.array(frames).shape, "pairs", domain.states)


if __name__ == "__main__":
    main()
