"""Host side of the reference GPU solve's extra keywords
(gpu_relative.py:67-101, :165-214): capture planes for centre distance,
rectangle contact and the local exit, probe stencils, and the argument
errors.  No GPU: every refusal here happens before a device is touched."""

import numpy as np
import pytest

from pursuit_evasion_b200.local_game.geometry import Footprint
from pursuit_evasion_b200.reversible.free_dp import (
    RelativeGrid,
    capture_plane,
    probe_stencils,
    solve,
)
from pursuit_evasion_b200.reversible.model import ReversibleConfig
from tests.helpers import A3, CONFIG1_GRID

BODIES = (Footprint(0.8, 0.5), Footprint(0.4, 0.25))
CONTACT = ReversibleConfig(point_vehicles=False, capture_rule="rectangle_contact")


def coords(grid):
    return -grid.extent + np.arange(grid.positions) * (2 * grid.extent / (grid.positions - 1))


def test_centre_distance_plane():
    c = coords(CONFIG1_GRID)
    plane = capture_plane(A3, CONFIG1_GRID)
    assert plane.shape == (17, 17) and plane.dtype == np.float32
    np.testing.assert_array_equal(
        plane, (np.hypot(c[:, None], c[None, :]) - A3.capture_radius).astype(np.float32))


def test_rectangle_contact_block_matches_oracle_separation(oracle):
    grid = RelativeGrid(13, 8, 3, 3, 3.0)
    block = capture_plane(CONTACT, grid, BODIES)
    assert block.shape == (8, 13, 13)
    c = coords(grid)
    psi = -np.pi + np.arange(8) * 2 * np.pi / 8
    for k in range(8):
        for iy in (0, 4, 6, 12):
            for ix in range(13):
                ref = oracle.rect_separation([0, 0, 0], [c[ix], c[iy], psi[k]], (0.8, 0.5),
                                             (0.4, 0.25))
                assert block[k, iy, ix] == pytest.approx(ref, abs=2e-7)
    assert (block <= 0).any() and (block > 0).any()


def test_exit_plane_holds_the_radius_outside():
    c = coords(CONFIG1_GRID)
    plane = capture_plane(A3, CONFIG1_GRID, exit_radius=2.5)
    outside = c[None, :] ** 2 + c[:, None] ** 2 > 2.5 ** 2
    assert outside.any() and (~outside).any()
    assert np.all(plane[outside] == np.float32(2.5))
    np.testing.assert_array_equal(plane[~outside], capture_plane(A3, CONFIG1_GRID)[~outside])
    block = capture_plane(CONTACT, CONFIG1_GRID, BODIES, exit_radius=2.5)
    assert np.all(block[:, outside] == np.float32(2.5))


def multilinear(field, grid, config, state):
    """Direct 2^5-corner interpolation of one (x, y, psi, vP, vE) state."""
    axes = grid.axes(config)
    q = [state[3], state[4], state[2], state[1], state[0]]
    lo, frac = [], []
    for k, (axis, n) in enumerate(zip(axes, grid.shape)):
        h = axis[1] - axis[0]
        if k == 2:
            f = ((q[k] + np.pi) % (2 * np.pi)) / h
            lo.append(int(np.floor(f)) % n)
            frac.append(f - np.floor(f))
        else:
            j = min(int(np.floor((q[k] - axis[0]) / h)), n - 2)
            lo.append(j)
            frac.append((q[k] - axis[0]) / h - j)
    total = 0.0
    for corner in range(32):
        idx, w = [], 1.0
        for k in range(5):
            bit = (corner >> k) & 1
            j = lo[k] + bit
            idx.append(j % grid.shape[k] if k == 2 else j)
            w *= frac[k] if bit else 1 - frac[k]
        total += w * float(field[tuple(idx)])
    return total


def test_probe_stencils_interpolate_like_a_direct_sum():
    grid = RelativeGrid(9, 6, 4, 3, 2.0)
    rng = np.random.default_rng(3)
    field = rng.standard_normal(grid.shape).astype(np.float32)
    (pmin, pmax), (emin, emax) = ((A3.pursuer.speed_min, A3.pursuer.speed_max),
                                  (A3.evader.speed_min, A3.evader.speed_max))
    states = np.column_stack([
        rng.uniform(-2, 2, 50), rng.uniform(-2, 2, 50), rng.uniform(-7, 7, 50),
        rng.uniform(pmin, pmax, 50), rng.uniform(emin, emax, 50)])
    states[0] = [2.0, -2.0, np.pi, pmax, emin]  # upper ends and the heading seam
    states[1] = [-2.0, 2.0, -np.pi, pmin, emax]
    kept, idx, w = probe_stencils(A3, grid, states)
    np.testing.assert_array_equal(kept, states)
    assert idx.shape == w.shape == (50, 32)
    np.testing.assert_allclose(w.sum(1), 1.0, atol=1e-12)
    got = (field.ravel()[idx] * w).sum(1)
    want = [multilinear(field, grid, A3, s) for s in states]
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("bad", [
    np.zeros((3, 4)), np.full((2, 5), np.nan), np.zeros((100001, 5)),
    [[9.0, 0, 0, 0, 0]], [[0, 0, 0, 5.0, 0]]])
def test_probe_validation(bad):
    with pytest.raises(ValueError):
        probe_stencils(A3, CONFIG1_GRID, bad)


def test_solve_refuses_bad_keywords_before_any_work(tmp_path):
    out = tmp_path / "t"
    with pytest.raises(ValueError, match="footprints"):
        solve(CONTACT, CONFIG1_GRID, out)
    with pytest.raises(ValueError, match="rectangle_contact"):
        solve(A3, CONFIG1_GRID, out, capture_footprints=BODIES)
    for r in (0.0, -1.0, 4.0, 5.0):
        with pytest.raises(ValueError, match="exit radius"):
            solve(A3, CONFIG1_GRID, out, exit_radius=r)
    with pytest.raises(ValueError, match="Probes"):
        solve(A3, CONFIG1_GRID, out, probes=np.zeros((2, 4)))
    assert not out.exists()


def test_solve_refuses_unknown_scheme_and_semi_lagrangian_extras(tmp_path):
    out = tmp_path / "t"
    with pytest.raises(ValueError, match="scheme"):
        solve(A3, CONFIG1_GRID, out, scheme="weno")
    with pytest.raises(ValueError, match="eno_lf"):
        solve(A3, CONFIG1_GRID, out, scheme="semi_lagrangian", tol=1e-3)
    with pytest.raises(ValueError, match="eno_lf"):
        solve(A3, CONFIG1_GRID, out, scheme="semi_lagrangian", exit_radius=2.0)
    assert not out.exists()
