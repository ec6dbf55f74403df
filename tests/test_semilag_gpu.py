"""Semi-Lagrangian min-max backup on the GPU (float32) against the FP64
oracle: values within float rounding, optimal action indices equal except
at ties, convergence of the minimum-time value iteration, warm starts, and
full-size properties on the 89M-cell grid."""

import numpy as np
import pytest

from pursuit_evasion_b200 import _native
from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
from pursuit_evasion_b200.reversible.semilag import (
    SemiLagrangianSolver,
    capture_time,
    interpolation_cfl_dt,
)
from tests import oracle_lib
from tests.helpers import A3, CONFIG1_GRID, CONFIG2_GRID

pytestmark = pytest.mark.gpu

# float32 value arithmetic vs the FP64 oracle, per backup
VALUE_ATOL = 2e-5
# an action index may differ only where the oracle's two candidates are
# this close (a tie within float rounding)
TIE_ATOL = 2e-4


def oracle_values(oracle, cfg, V, cell, grid):
    """values[up, ue] (FP64) at one cell: the interpolated value at the
    successor of every pursuer / evader action pair."""
    iv, ie, ip, iy, ix = np.unravel_index(cell, grid.shape)
    axes = grid.axes(A3)
    state = (axes[4][ix], axes[3][iy], axes[2][ip], axes[0][iv], axes[1][ie])
    vals = np.array([[oracle.sl_interpolate(cfg, V, oracle.sl_successor(cfg, state, up, ue))
                      for ue in range(9)] for up in range(9)])
    if cfg.mode == oracle_lib.SL_MINTIME:
        vals = np.clip(vals, 0, 1)
    return vals


def oracle_worst(oracle, cfg, V, cell, grid):
    """Per pursuer action, the max over evader actions (FP64) at one cell."""
    return oracle_values(oracle, cfg, V, cell, grid).max(axis=1)


@pytest.mark.parametrize("mode", ["tube", "min_time"])
def test_single_backup_matches_oracle(oracle, mode):
    grid = RelativeGrid(13, 12, 7, 7, 3.0)
    dt = interpolation_cfl_dt(A3, grid)
    omode = oracle_lib.SL_TUBE if mode == "tube" else oracle_lib.SL_MINTIME
    cfg = oracle.sl_cfg(A3, grid, dt, omode)
    rng = np.random.default_rng(5)
    if mode == "tube":
        V = oracle.sl_init(cfg, grid.states) + 0.05 * rng.normal(size=grid.states)
    else:
        V = rng.uniform(0, 1, grid.states)
    V32 = V.astype(np.float32)
    ref, pp, pe = oracle.sl_backup(cfg, V32.astype(np.float64), with_policy=True)
    with SemiLagrangianSolver(A3, grid, dt=dt, mode=mode) as s:
        s.initialize(V32)
        s.backup(with_policy=True)
        got = s.value().ravel()
        gp, ge = (a.ravel() for a in s.policy())
    np.testing.assert_allclose(got, ref, atol=VALUE_ATOL, rtol=0)
    V64 = V32.astype(np.float64)
    # every pursuer index that differs is a tie of the oracle's own values
    mismatch = np.flatnonzero(gp != pp)
    assert len(mismatch) < 0.01 * grid.states
    for cell in mismatch:
        worst = oracle_worst(oracle, cfg, V64, cell, grid)
        assert abs(worst[gp[cell]] - worst[pp[cell]]) <= TIE_ATOL
    # where the pursuer indices agree, every evader index that differs is a
    # tie among that pursuer action's replies
    e_mismatch = np.flatnonzero((gp == pp) & (ge != pe))
    assert len(e_mismatch) < 0.02 * grid.states
    for cell in e_mismatch:
        vals = oracle_values(oracle, cfg, V64, cell, grid)[pp[cell]]
        assert abs(vals[ge[cell]] - vals[pe[cell]]) <= TIE_ATOL


@pytest.mark.parametrize("mode", ["tube", "min_time"])
def test_policy_follows_the_reference_tie_rules_on_exact_ties(oracle, mode):
    """A field that depends on the pursuer's speed only: all evader replies
    tie exactly (the evader takes the neutral action first,
    map_game_policy.py:12-18), and the three curvatures of the best
    acceleration tie (the pursuer takes the smallest (|k|, |a|, index),
    controllers.py:122-126).  GPU and oracle pick the same actions
    everywhere."""
    grid = RelativeGrid(13, 12, 7, 7, 3.0)
    dt = interpolation_cfl_dt(A3, grid)
    omode = oracle_lib.SL_TUBE if mode == "tube" else oracle_lib.SL_MINTIME
    cfg = oracle.sl_cfg(A3, grid, dt, omode)

    def policies(V32):
        _, pp, pe = oracle.sl_backup(cfg, V32.ravel().astype(np.float64), with_policy=True)
        with SemiLagrangianSolver(A3, grid, dt=dt, mode=mode) as s:
            s.initialize(V32.ravel())
            s.backup(with_policy=True)
            gp, ge = (a.ravel() for a in s.policy())
        return gp, ge, pp, pe

    # all 81 pairs tie exactly (a zero field): both players hold course
    gp, ge, pp, pe = policies(np.zeros(grid.states, np.float32))
    assert np.all(gp == 4) and np.all(pp == 4) and np.all(ge == 4) and np.all(pe == 4)

    # values small enough that the float32 blend of the speed corners stays
    # well inside the 1e-7 tie tolerance
    level = np.linspace(0.1, 0.3, grid.p_speeds) ** 2  # increasing in vP
    V32 = np.broadcast_to(level[:, None, None, None, None], grid.shape).astype(np.float32)
    gp, ge, pp, pe = policies(V32)
    np.testing.assert_array_equal(gp, pp)
    np.testing.assert_array_equal(ge, pe)
    assert np.all(ge == 4)            # neutral reply
    assert np.all(gp % 3 == 1)        # straight ahead: |k| = 0
    # slowest successor speed: brake, except at the lowest speed level where
    # braking and holding give the same speed and |a| = 0 wins
    iv = np.unravel_index(np.arange(grid.states), grid.shape)[0]
    assert np.all(gp[iv > 0] == 1) and np.all(gp[iv == 0] == 4)


@pytest.mark.parametrize("mode", ["tube", "min_time"])
@pytest.mark.parametrize("grid", [RelativeGrid(13, 12, 7, 7, 3.0),
                                  RelativeGrid(21, 16, 5, 9, 5.0)])
def test_tiled_value_backup_matches_oracle(oracle, mode, grid):
    """The shared-memory tiled kernel (value-only backups) on random fields."""
    dt = interpolation_cfl_dt(A3, grid)
    omode = oracle_lib.SL_TUBE if mode == "tube" else oracle_lib.SL_MINTIME
    cfg = oracle.sl_cfg(A3, grid, dt, omode)
    rng = np.random.default_rng(11)
    if mode == "tube":
        V = oracle.sl_init(cfg, grid.states) + 0.05 * rng.normal(size=grid.states)
    else:
        V = rng.uniform(0, 1, grid.states)
    V32 = V.astype(np.float32)
    ref = oracle.sl_backup(cfg, V32.astype(np.float64))
    with SemiLagrangianSolver(A3, grid, dt=dt, mode=mode) as s:
        s.set_kernel("tiled")
        assert s.kernel == "tiled"
        s.initialize(V32)
        s.backup()
        got = s.value().ravel()
        residual = s.residual()
        evaluations = s.evaluations()
    np.testing.assert_allclose(got, ref, atol=VALUE_ATOL, rtol=0)
    assert residual == pytest.approx(float(np.abs(got - V32).max()), rel=1e-6, abs=1e-12)
    # every live cell probes the 9 pursuer actions; none evaluates more than
    # the 81 pairs (cells inside the capture disk are not live in min_time)
    live = grid.states if mode == "tube" else int(np.count_nonzero(ref > 0))
    assert 9 * live <= evaluations <= 81 * grid.states


@pytest.mark.parametrize("mode", ["tube", "min_time"])
def test_tiled_and_generic_kernels_agree_over_iterations(mode):
    """Ten value-only backups with the tiled kernel (pruned, hint-ordered)
    and with the generic kernel: the same fields up to float rounding."""
    grid = RelativeGrid(33, 24, 7, 7, 6.0)
    out = {}
    for kernel in ("tiled", "generic"):
        with SemiLagrangianSolver(A3, grid, mode=mode) as s:
            s.set_kernel(kernel)
            assert s.kernel == kernel
            s.initialize()
            s.iterate(10, tol=0.0, check_every=10)
            out[kernel] = s.value().ravel().copy()
    np.testing.assert_allclose(out["tiled"], out["generic"], atol=10 * VALUE_ATOL, rtol=0)


def test_tiled_kernel_refused_where_it_does_not_apply():
    grid = RelativeGrid(13, 12, 7, 7, 3.0)
    big_dt = 4 * interpolation_cfl_dt(A3, grid)  # successors several cells away
    with SemiLagrangianSolver(A3, grid, dt=big_dt, mode="tube") as s:
        assert s.kernel == "generic"
        with pytest.raises(ValueError):
            s.set_kernel("tiled")


def test_tube_backups_are_monotone_and_track_oracle(oracle):
    grid = CONFIG1_GRID
    dt = interpolation_cfl_dt(A3, grid)
    cfg = oracle.sl_cfg(A3, grid, dt, oracle_lib.SL_TUBE)
    V = oracle.sl_init(cfg, grid.states)
    with SemiLagrangianSolver(A3, grid, dt=dt, mode="tube") as s:
        s.initialize()
        first = s.value().ravel().copy()
        np.testing.assert_array_equal(first, V.astype(np.float32))
        for _ in range(4):
            V = oracle.sl_backup(cfg, V)
        iters, residual, _ = s.iterate(4, tol=0.0)
        got = s.value().ravel()
    assert iters == 4
    assert np.all(got <= first)
    np.testing.assert_allclose(got, V, atol=4 * VALUE_ATOL, rtol=0)


def test_min_time_iteration_converges_and_warm_start_is_a_fixed_point(oracle):
    grid = RelativeGrid(11, 8, 5, 5, 3.0)
    dt = 0.1
    cfg = oracle.sl_cfg(A3, grid, dt, oracle_lib.SL_MINTIME)
    with SemiLagrangianSolver(A3, grid, dt=dt, mode="min_time") as s:
        s.initialize()
        iters, residual, converged = s.iterate(2000, tol=1e-5, check_every=1)
        u = s.value().ravel().copy()
    assert converged and residual < 1e-5
    # the oracle, started from the GPU's converged field, barely moves it
    step = oracle.sl_backup(cfg, u.astype(np.float64))
    assert np.abs(step - u).max() < 5e-5
    # captured cells hold 0, capture times are finite and positive elsewhere
    T = capture_time(u)
    assert np.all(T[u == 0] == 0)
    assert np.isfinite(T).mean() > 0.5
    # a warm start at the fixed point converges at once
    with SemiLagrangianSolver(A3, grid, dt=dt, mode="min_time") as s:
        s.initialize(u)
        iters2, residual2, converged2 = s.iterate(50, tol=1e-5, check_every=1)
    assert converged2 and iters2 <= 2


def test_full_size_backup_spot_checks(oracle):
    """89,434,800 cells, one tube backup: 400 sampled cells against the FP64
    oracle, monotone, finite, policy recorded."""
    grid = CONFIG2_GRID
    dt = interpolation_cfl_dt(A3, grid)
    cfg = oracle.sl_cfg(A3, grid, dt, oracle_lib.SL_TUBE)
    launches = _native.launch_count()
    with SemiLagrangianSolver(A3, grid, dt=dt, mode="tube") as s:
        s.initialize()
        v0 = s.value().ravel().copy()
        s.backup(with_policy=True)
        v1 = s.value().ravel()
        gp, _ = s.policy()
    assert _native.launch_count() - launches >= 2
    assert np.isfinite(v1).all() and np.all(v1 <= v0)
    rng = np.random.default_rng(8)
    cells = rng.choice(grid.states, size=400, replace=False)
    ref, pp, _ = oracle.sl_backup_cells(cfg, v0.astype(np.float64), cells)
    np.testing.assert_allclose(v1[cells], ref, atol=VALUE_ATOL, rtol=0)
    agree = np.mean(gp.ravel()[cells] == pp)
    assert agree > 0.95


def test_full_size_tiled_backup_spot_checks(oracle):
    """89,434,800 cells, two value-only backups with the tiled kernel (the
    second one pruned with the first one's hints): sampled cells against the
    FP64 oracle."""
    grid = CONFIG2_GRID
    dt = interpolation_cfl_dt(A3, grid)
    cfg = oracle.sl_cfg(A3, grid, dt, oracle_lib.SL_TUBE)
    rng = np.random.default_rng(9)
    cells = rng.choice(grid.states, size=300, replace=False)
    with SemiLagrangianSolver(A3, grid, dt=dt, mode="tube") as s:
        assert s.kernel == "tiled"
        s.initialize()
        s.backup()
        v1 = s.value().ravel().copy()
        s.backup()
        v2 = s.value().ravel()
    v0 = oracle.sl_init(cfg, grid.states)
    ref1, _, _ = oracle.sl_backup_cells(cfg, v0, cells)
    np.testing.assert_allclose(v1[cells], ref1, atol=VALUE_ATOL, rtol=0)
    ref2, _, _ = oracle.sl_backup_cells(cfg, v1.astype(np.float64), cells)
    np.testing.assert_allclose(v2[cells], ref2, atol=VALUE_ATOL, rtol=0)
    assert np.isfinite(v2).all() and np.all(v2 <= v1)


@pytest.mark.parametrize("mode", ["tube", "min_time"])
def test_work_skipping_is_exact(mode):
    """Tiled value iteration with and without work skipping: the same
    residual sequence and iteration count, bit-identical fields, and never
    more items computed with skipping (items whose neighbourhood did not
    change are copied).  How many are skipped depends on the field: the
    tube field (a distance) moves everywhere on every backup, and in
    minimum-time mode the interpolated constant 1 ahead of the front lands
    within an ulp of 1, so those cells still change in their last bit."""
    grid = RelativeGrid(33, 24, 7, 7, 6.0)
    out = {}
    for skip in (False, True):
        with SemiLagrangianSolver(A3, grid, mode=mode) as s:
            s.set_kernel("tiled")
            s.set_skip(skip)
            s.initialize()
            iters, residual, converged = s.iterate(600, tol=1e-5, check_every=5)
            items = s.tile["items"]
            out[skip] = (s.value().copy(), iters, residual, s.items_computed())
    assert out[True][1] == out[False][1] and out[True][2] == out[False][2]
    np.testing.assert_array_equal(out[True][0].view(np.uint32), out[False][0].view(np.uint32))
    assert out[False][3] == items * out[False][1]
    assert out[True][3] <= out[False][3]
