"""Relative 5D ENO/LF solve on the GPU against the oracle and the reference.

* exact path (double local, no contraction): bit for bit equal to the oracle,
  the reference executable and the golden vectors, every frame and arrival;
* fast path (float32 local): within float rounding of the oracle;
* drop-in solve(): the table directory reads back through RelativeTable;
* full-size properties on the 89M-cell grid: the tube never increases, the
  fast and exact paths agree, and the capture disk keeps arrival 0.
"""

import shutil

import numpy as np
import pytest

from pursuit_evasion_b200 import _native
from pursuit_evasion_b200.reversible.free_dp import RelativeGrid, solve
from pursuit_evasion_b200.reversible.relative_solver import RelativeSolver
from pursuit_evasion_b200.reversible.relative_table import RelativeTable
from tests import oracle_lib
from tests.helpers import A3, CONFIG1_GRID, CONFIG2_GRID, DEFAULT, bits, relative_goldens

pytestmark = pytest.mark.gpu

GOLDEN = relative_goldens()
# Float32 local arithmetic against the double-local oracle: values are O(1-10)
# and each stage rounds in float; observed differences stay below these.
FAST_ATOL = 2e-5
FAST_RTOL = 2e-6


def gpu_frames(config, grid, horizon, output_dt, order, precision):
    times = np.minimum(np.arange(int(np.ceil(horizon / output_dt - 1e-10)) + 1)
                       * output_dt, horizon)
    frames = []
    with RelativeSolver(config, grid, order=order,
                        local_precision=precision) as s:
        s.initialize()
        frames.append(s.field().copy())
        for goal in times[1:]:
            s.advance(goal)
            frames.append(s.field().copy())
        return np.array(frames), s.arrival().copy(), s.steps


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_exact_path_reproduces_reference_golden_bitwise(name):
    case = GOLDEN[name]
    frames, arrival, steps = gpu_frames(case["config"], case["grid"],
                                        case["horizon"], case["output_dt"],
                                        case["order"], "float64")
    assert steps == case["internal_steps"]
    np.testing.assert_array_equal(bits(frames), bits(case["frames"]))
    np.testing.assert_array_equal(bits(arrival), bits(case["arrival"]))


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_fast_path_matches_reference_golden_within_float_rounding(name):
    case = GOLDEN[name]
    frames, arrival, steps = gpu_frames(case["config"], case["grid"],
                                        case["horizon"], case["output_dt"],
                                        case["order"], "float32")
    assert steps == case["internal_steps"]
    np.testing.assert_allclose(frames, case["frames"], atol=FAST_ATOL,
                               rtol=FAST_RTOL)
    ref = case["arrival"]
    assert np.array_equal(np.isnan(arrival), np.isnan(ref)) or (
        np.mean(np.isnan(arrival) != np.isnan(ref)) < 1e-3)


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("config", [A3, DEFAULT], ids=["a3", "default"])
def test_exact_path_matches_oracle_on_readme_grid(oracle, order, config):
    cfg = oracle.rel_cfg(config, CONFIG1_GRID, order=order)
    ref_frames, ref_arrival, ref_steps = oracle.rel_solve_f32(cfg, 0.2, 0.1)
    frames, arrival, steps = gpu_frames(config, CONFIG1_GRID, 0.2, 0.1, order,
                                        "float64")
    assert steps == ref_steps
    np.testing.assert_array_equal(bits(frames.reshape(ref_frames.shape)),
                                  bits(ref_frames))
    np.testing.assert_array_equal(bits(arrival.ravel()), bits(ref_arrival))


@pytest.mark.parametrize("order", [1, 2])
def test_fast_path_matches_oracle_on_readme_grid(oracle, order):
    cfg = oracle.rel_cfg(A3, CONFIG1_GRID, order=order)
    ref_frames, _, _ = oracle.rel_solve_f32(cfg, 0.2, 0.1)
    frames, _, _ = gpu_frames(A3, CONFIG1_GRID, 0.2, 0.1, order, "float32")
    np.testing.assert_allclose(frames.reshape(ref_frames.shape), ref_frames,
                               atol=FAST_ATOL, rtol=FAST_RTOL)


@pytest.mark.skipif(not oracle_lib.REF_RELATIVE.exists(),
                    reason="reference executable not built (make -C oracle ref)")
def test_solve_table_equals_reference_executable_table(tmp_path):
    """README smoke test: same call, same files, same bits."""
    meta = solve(A3, CONFIG1_GRID, tmp_path / "gpu", horizon=0.2)
    folder, timing = oracle_lib.run_reference_relative(A3, CONFIG1_GRID,
                                                       horizon=0.2,
                                                       output_dt=0.1)
    try:
        assert meta["status"] == "complete"
        assert meta["internal_steps"] == timing["internal_steps"]
        assert meta["cfl_dt_limit"] == pytest.approx(timing["cfl_dt_limit"], rel=1e-12)
        for name in ("fields.f32", "final.f32", "arrival.f32"):
            ours = np.fromfile(tmp_path / "gpu" / name, np.uint32)
            theirs = np.fromfile(folder / name, np.uint32)
            np.testing.assert_array_equal(ours, theirs, err_msg=name)
    finally:
        shutil.rmtree(folder)
    table = RelativeTable(tmp_path / "gpu", A3)
    state = np.array([[0.2, 0.1, 0.0, 1.0, 0.5], [1.2, -0.3, 2.0, 0.4, -0.2]])
    t = table.value(state)
    assert t[0] == 0 and (np.isnan(t[1]) or 0 < t[1] <= 0.2)
    with pytest.raises(FileExistsError):
        solve(A3, CONFIG1_GRID, tmp_path / "gpu", horizon=0.2)


def test_solve_fast_path_with_convergence_tolerance(tmp_path):
    meta = solve(A3, RelativeGrid(9, 8, 7, 7, 1.0), tmp_path / "tol",
                 horizon=5.0, output_dt=0.5, local_precision="float32",
                 tol=1e-4)
    assert meta["status"] == "complete"
    table = RelativeTable(tmp_path / "tol", A3)
    assert table.horizon == meta["converged_time"] < 5.0
    assert np.all(np.diff(table.fields, axis=0) <= 0)


def test_full_size_grid_properties():
    """89,434,800 cells: a few RK2 steps on both paths.  The tube never rises,
    the capture disk keeps arrival 0, the two paths agree to float rounding,
    and the reported residual is the sup-norm change of the last step."""
    grid = CONFIG2_GRID
    launches = _native.launch_count()
    with RelativeSolver(A3, grid, local_precision="float32") as fast, \
            RelativeSolver(A3, grid, local_precision="float64") as exact:
        fast.initialize()
        exact.initialize()
        v0 = fast.field().copy()
        dt = fast.cfl_dt_limit
        for _ in range(3):
            fast.step(dt)
            exact.step(dt)
        before_last = fast.field().copy()
        fast.step(dt)
        exact.step(dt)
        v_fast = fast.field().copy()
        v_exact = exact.field().copy()
        residual, increase = fast.stats()
        arrival = fast.arrival()
    assert _native.launch_count() - launches >= 16
    assert np.isfinite(v_fast).all()
    assert np.all(v_fast <= v0)
    assert increase == 0.0
    np.testing.assert_allclose(v_fast, v_exact, atol=1e-4, rtol=1e-5)
    change = np.abs(v_fast.astype(np.float64) - before_last).max()
    assert residual == pytest.approx(change, rel=1e-6)
    assert np.all(arrival[v0 <= 0] == 0)
