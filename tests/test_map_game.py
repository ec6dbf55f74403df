"""Host side of the 8D obstacle map game driver (gpu_map_game.py
restatement): the 2^8-corner interpolation stencil and the argument errors,
which all come before any device work."""

import numpy as np
import pytest

from pursuit_evasion_b200.reversible.gpu_map_game import interpolation_stencil, solve
from pursuit_evasion_b200.reversible.model import ReversibleConfig
from pursuit_evasion_b200.reversible.world_dp import WorldGrid

MAP = ReversibleConfig(point_vehicles=False)
GRID = WorldGrid(7, 6, 4, 3, 3.0)


def clear(grid):
    z = np.zeros((grid.positions, grid.positions, grid.headings), np.float32)
    return z + 1, z + 1


def test_stencil_reproduces_multilinear_functions():
    axes = GRID.axes(MAP)
    rng = np.random.default_rng(0)
    lo = np.array([a[0] for a in axes])
    hi = np.array([a[-1] for a in axes])
    states = lo + (hi - lo) * rng.random((40, 8))
    states[0] = hi  # upper ends
    idx, w, valid = interpolation_stencil(states, axes, (2, 6))
    assert valid.all() and idx.shape == (40, 256)
    np.testing.assert_allclose(w.sum(1), 1, atol=1e-12)
    # a function linear in each non-periodic axis, constant in the headings
    mesh = np.meshgrid(*axes, indexing="ij")
    coef = [0.3, -0.7, 0, 1.1, 0.5, 0.2, 0, -0.4]
    f = sum(c * m for c, m in zip(coef, mesh)).ravel()
    np.testing.assert_allclose((f[idx] * w).sum(1), states @ np.array(coef), atol=1e-9)
    # headings wrap: a state beyond the last heading node uses node 0
    s = states[1].copy()
    s[2] = axes[2][-1] + 0.5 * (axes[2][1] - axes[2][0])
    i2, w2, _ = interpolation_stencil(s[None], axes, (2, 6))
    nodes = np.unravel_index(i2[0][w2[0] > 0], GRID.shape)[2]
    assert set(nodes) == {len(axes[2]) - 1, 0}
    bad = states[:1].copy()
    bad[0, 0] = hi[0] + 1
    assert not interpolation_stencil(bad, axes, (2, 6))[2][0]


def test_solve_argument_errors(tmp_path):
    with pytest.raises(ValueError, match="point_vehicles"):
        solve(ReversibleConfig(), GRID, clear(GRID), tmp_path / "a")
    with pytest.raises(TypeError):
        solve(MAP, GRID, object(), tmp_path / "b")
    with pytest.raises(ValueError, match="order1/2"):
        solve(MAP, GRID, clear(GRID), tmp_path / "c", cfl=1.5)
    with pytest.raises(ValueError, match="node indices"):
        solve(MAP, GRID, clear(GRID), tmp_path / "d", query_indices=[GRID.states])
    with pytest.raises(ValueError, match="OR"):
        solve(MAP, GRID, clear(GRID), tmp_path / "e", query_indices=[0],
              query_states=np.zeros((1, 8)))
    with pytest.raises(ValueError, match="outside"):
        solve(MAP, GRID, clear(GRID), tmp_path / "f", query_states=np.full((1, 8), 9.0))
