"""free_dp.solve(scheme="semi_lagrangian"): the relative table filled by
the semi-Lagrangian tube backup.  Frames against the FP64 oracle backup
(oracle/semilag5d.c) with the same held-command steps, arrival times
against the frames, and the policy files against a direct solver run."""

import json

import numpy as np
import pytest

from pursuit_evasion_b200.reversible.free_dp import output_times, probe_stencils, solve
from pursuit_evasion_b200.reversible.semilag import SemiLagrangianSolver, interpolation_cfl_dt
from tests import oracle_lib
from tests.helpers import A3, CONFIG1_GRID
from tests.test_semilag_gpu import VALUE_ATOL

pytestmark = pytest.mark.gpu


def segments(times, output_dt, limit):
    """(step dt, backups) per output interval, as the solve splits them."""
    out = []
    for a, b in zip(times[:-1], times[1:]):
        length = output_dt if abs((b - a) - output_dt) <= 1e-9 * max(1, output_dt) else b - a
        n = max(1, int(np.ceil(length / limit - 1e-9)))
        out.append((length / n, n))
    return out


def test_semi_lagrangian_table_tracks_oracle(oracle, tmp_path):
    grid, horizon, output_dt = CONFIG1_GRID, 0.25, 0.1
    rng = np.random.default_rng(4)
    states = np.column_stack([rng.uniform(-3, 3, 20), rng.uniform(-3, 3, 20),
                              rng.uniform(-3, 3, 20), rng.uniform(-1, 2, 20),
                              rng.uniform(-0.5, 1, 20)])
    meta = solve(A3, grid, tmp_path / "t", horizon=horizon, output_dt=output_dt,
                 scheme="semi_lagrangian", probes=states)
    times = output_times(horizon, output_dt)
    limit = interpolation_cfl_dt(A3, grid)
    plan = segments(times, output_dt, limit)
    assert meta["status"] == "complete" and meta["scheme"] == "semi_lagrangian"
    assert meta["internal_steps"] == sum(n for _, n in plan)
    assert json.loads((tmp_path / "t" / "meta.json").read_text())["status"] == "complete"
    N = grid.states
    frames = np.fromfile(tmp_path / "t" / "fields.f32", np.float32).reshape(len(times), N)
    # FP64 oracle with the same steps
    V = oracle.sl_init(oracle.sl_cfg(A3, grid, plan[0][0], oracle_lib.SL_TUBE), N)
    np.testing.assert_array_equal(frames[0], V.astype(np.float32))
    backups = 0
    for k, (dt, n) in enumerate(plan, start=1):
        cfg = oracle.sl_cfg(A3, grid, dt, oracle_lib.SL_TUBE)
        for _ in range(n):
            V = oracle.sl_backup(cfg, V)
        backups += n
        np.testing.assert_allclose(frames[k], V, atol=backups * VALUE_ATOL, rtol=0)
        assert np.all(frames[k] <= frames[k - 1])
    # arrival: inside the interval in which the cell's value crossed zero
    arrival = np.fromfile(tmp_path / "t" / "arrival.f32", np.float32)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "t" / "final.f32", np.float32),
                                  frames[-1])
    assert np.array_equal(np.isfinite(arrival), frames[-1] <= 0)
    assert np.all(arrival[frames[0] <= 0] == 0)
    for k in range(1, len(times)):
        crossed = (frames[k - 1] > 0) & (frames[k] <= 0)
        assert np.all((arrival[crossed] > times[k - 1] - 1e-6)
                      & (arrival[crossed] <= times[k] + 1e-6))
    # probes and residuals
    probes = np.fromfile(tmp_path / "t" / "probes.f64").reshape(len(times), 20)
    _, idx, w = probe_stencils(A3, grid, states)
    np.testing.assert_allclose(probes, (frames[:, idx].astype(np.float64) * w).sum(-1),
                               rtol=1e-12, atol=1e-12)
    residuals = np.fromfile(tmp_path / "t" / "residuals.f64")
    assert residuals.shape == (len(times) - 1,) and np.all(residuals >= 0)
    # the policy files are the last backup's optimal actions
    pol_p = np.fromfile(tmp_path / "t" / "policy_p.u8", np.uint8)
    pol_e = np.fromfile(tmp_path / "t" / "policy_e.u8", np.uint8)
    assert pol_p.size == pol_e.size == N and pol_p.max() < 9 and pol_e.max() < 9
    dt, n = plan[-1]
    with SemiLagrangianSolver(A3, grid, dt=dt, mode="tube") as s:
        s.initialize(frames[-2])
        for k in range(n):
            s.backup(with_policy=k == n - 1)
        p, e = s.policy()
        np.testing.assert_allclose(s.value().ravel(), frames[-1], atol=VALUE_ATOL, rtol=0)
    assert np.mean(p.ravel() != pol_p) < 1e-3 and np.mean(e.ravel() != pol_e) < 1e-3
