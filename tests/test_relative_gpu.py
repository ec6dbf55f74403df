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
# Float32 local arithmetic against the double-local oracle.  The bulk of the
# cells agree to float rounding (FAST_ATOL + FAST_RTOL*|v|).  ENO2 picks the
# smaller of two second differences; where the two are tied to rounding, float
# and double arithmetic can pick differently, which moves that slope by
# h*(D2_a - D2_b)/2.  Such flips touch well under 0.1 % of the cells and stay
# below FLIP_MAX -- the same size as the reference executable's own float32
# storage differs from a float64-storage solve (tests/test_oracle.py).
FAST_ATOL = 2e-5
FAST_RTOL = 2e-6
FLIP_FRACTION = 1e-3
FLIP_MIN_COUNT = 4
FLIP_MAX = 1e-3


def assert_fast_close(actual, expected):
    actual = np.asarray(actual, np.float64).ravel()
    expected = np.asarray(expected, np.float64).ravel()
    diff = np.abs(actual - expected)
    outside = diff > FAST_ATOL + FAST_RTOL * np.abs(expected)
    assert outside.sum() <= max(FLIP_MIN_COUNT, FLIP_FRACTION * outside.size), (
        outside.sum(), diff.max())
    assert diff.max() <= FLIP_MAX, diff.max()


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
    assert_fast_close(frames, case["frames"])
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
    assert_fast_close(frames, ref_frames)


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


def test_solve_stops_at_first_step_below_tolerance(oracle, tmp_path):
    """tol: the solve ends after the first RK2 step whose sup-norm change is
    below tol.  The exact path shares the oracle's bits, so the oracle's
    residual sequence predicts the stopping step exactly."""
    grid = RelativeGrid(9, 8, 7, 7, 1.0)
    cfg = oracle.rel_cfg(A3, grid)
    a, arrival = np.empty(grid.states, np.float32), np.empty(grid.states, np.float32)
    import ctypes
    oracle.lib.po_rel_init(ctypes.addressof(cfg), a.ctypes.data, arrival.ctypes.data)
    b = np.empty_like(a)
    dt = oracle.rel_cfl_limit(cfg)
    residuals, t = [], 0.0
    for _ in range(40):
        old = a.copy()
        oracle.rel_stage_f32(cfg, a, b, arrival, dt, t, 0)
        oracle.rel_stage_f32(cfg, b, a, arrival, dt, t, 1)
        t += dt
        residuals.append(np.abs(a.astype(np.float64) - old).max())
    tol = sorted(residuals)[4] * (1 + 1e-9)
    first = next(k for k, r in enumerate(residuals) if r < tol) + 1
    meta = solve(A3, grid, tmp_path / "tol", horizon=40 * dt, output_dt=40 * dt,
                 tol=tol)
    assert meta["internal_steps"] == first
    assert meta["converged_time"] == pytest.approx(first * dt, rel=1e-12)
    table = RelativeTable(tmp_path / "tol", A3)
    assert table.horizon == meta["converged_time"]
    assert len(table.times) == 2


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


def test_history_written_while_solving_equals_synchronous_frames(tmp_path):
    """fields.f32 from the asynchronous history writer (device snapshots, two
    slots, a writer thread) holds, in order, exactly the frames a stopped
    solver copies out synchronously, also when frames queue up."""
    grid = RelativeGrid(9, 8, 7, 7, 1.0)
    times = np.round(np.arange(0, 21) * 0.025, 10)
    meta = solve(A3, grid, tmp_path / "h", horizon=float(times[-1]), output_dt=0.025)
    assert meta["frames"] == len(times)
    written = np.fromfile(tmp_path / "h" / "fields.f32", np.float32).reshape(len(times), -1)
    with RelativeSolver(A3, grid, local_precision="float64") as s:  # solve's default
        s.initialize()
        expected = [s.field().ravel().copy()]
        for goal in times[1:]:
            s.advance(float(goal))
            expected.append(s.field().ravel().copy())
    np.testing.assert_array_equal(written.view(np.uint32), np.array(expected).view(np.uint32))


@pytest.mark.parametrize("positions", [10, 11, 12, 13])
def test_fast_path_x_end_rules_for_every_row_length(oracle, positions):
    """The float32 stage places its x end rules by nx mod 4 (one compiled
    variant per residue): each residue tracks the double-local oracle."""
    grid = RelativeGrid(positions, 8, 5, 4, 3.0)
    cfg = oracle.rel_cfg(A3, grid)
    ref_frames, _, ref_steps = oracle.rel_solve_f32(cfg, 0.2, 0.1)
    frames, _, steps = gpu_frames(A3, grid, 0.2, 0.1, 2, "float32")
    assert steps == ref_steps
    assert_fast_close(frames, ref_frames)


def test_fast_path_does_not_depend_on_the_tile():
    """Each cell's float32 update is the same arithmetic whatever the work
    item (rows per item, headings per item): results are bit-identical over
    tiles, including one-row items and four-heading items, and tiles whose
    last heading chunk is shorter than four headings are refused."""
    grid = RelativeGrid(17, 12, 7, 7, 4.0)
    results = []
    for tile in (None, (1, 4), (5, 6), (17, 12), (3, 8)):
        with RelativeSolver(A3, grid, local_precision="float32") as s:
            if tile is not None:
                s.set_tile(*tile)
                assert s.tile[:2] == tile
            s.initialize()
            s.advance(0.15)
            results.append((s.field().copy(), s.arrival().copy()))
    for field, arrival in results[1:]:
        np.testing.assert_array_equal(bits(field), bits(results[0][0]))
        np.testing.assert_array_equal(bits(arrival), bits(results[0][1]))
    with RelativeSolver(A3, grid, local_precision="float32") as s:
        with pytest.raises(ValueError):
            s.set_tile(4, 5)  # 12 headings = 5 + 5 + 2: a 2-heading item


@pytest.mark.parametrize("name", sorted(GOLDEN)[:2] + ["readme-o1", "readme-o2"])
def test_fp64_storage_solve_equals_fp64_oracle_bitwise(oracle, name):
    """The FP64-storage solve (the exact stage with double values, which
    measures float32 tables at full size) equals the CPU FP64 oracle
    po_rel_stage_f64 bit for bit, frame driver included."""
    from pursuit_evasion_b200.reversible.fp64_table import RelativeSolverF64

    if name.startswith("readme"):
        config, grid, horizon, output_dt = A3, CONFIG1_GRID, 0.2, 0.1
        order = int(name[-1])
    else:
        case = GOLDEN[name]
        config, grid = case["config"], case["grid"]
        horizon, output_dt, order = case["horizon"], case["output_dt"], case["order"]
    final, steps = oracle.rel_solve_f64(oracle.rel_cfg(config, grid, order=order), horizon,
                                        output_dt)
    times = np.minimum(np.arange(1, int(np.ceil(horizon / output_dt - 1e-10)) + 1)
                       * output_dt, horizon)
    with RelativeSolverF64(config, grid, order=order) as s:
        s.initialize()
        for goal in times:
            s.advance(goal)
        got = s.field().ravel()
        assert s.steps == steps
        assert s.residual() > 0
    np.testing.assert_array_equal(got.view(np.uint64), final.view(np.uint64))


def test_fp64_table_error_of_float32_tables_on_the_subsampled_tile(oracle):
    """On a 33x24x9x9 grid over 0.5 s: the FP64-storage solve equals the
    CPU FP64 oracle bit for bit, the reference-arithmetic float32 table's
    error against it (every 2nd x, y, psi; all speeds) equals the oracle's
    own float32-vs-FP64 error, and the float32-local table stays within
    twice that error (max 4.7e-4, mean 1.3e-6 for the reference
    arithmetic)."""
    from pursuit_evasion_b200.reversible.fp64_table import RelativeSolverF64, subsampled_error

    grid = RelativeGrid(33, 24, 9, 9, 6.0)
    cfg = oracle.rel_cfg(A3, grid)
    frames, _, _ = oracle.rel_solve_f32(cfg, 0.5, 0.5)
    final64, _ = oracle.rel_solve_f64(cfg, 0.5, 0.5)
    with RelativeSolverF64(A3, grid) as r:
        r.initialize()
        r.advance(0.5)
        ref = r.field()
    np.testing.assert_array_equal(ref.ravel().view(np.uint64), final64.view(np.uint64))
    expected = subsampled_error(frames[-1].reshape(grid.shape), ref, step=2)
    errors = {}
    for precision in ("float64", "float32"):
        with RelativeSolver(A3, grid, local_precision=precision) as s:
            s.initialize()
            s.advance(0.5)
            errors[precision] = subsampled_error(s.field(), ref, step=2)
    assert errors["float64"] == expected
    assert expected["nodes"] == 9 * 9 * 12 * 17 * 17
    assert errors["float32"]["max_abs"] <= 2 * expected["max_abs"]
    assert errors["float32"]["mean_abs"] <= 2 * expected["mean_abs"]


def test_compile_time_tile_equals_the_general_kernel():
    """On 65-position grids the default 13-row tile runs a variant with
    compile-time offsets; any other tile runs the general kernel.  Both give
    the same bits."""
    grid = RelativeGrid(65, 8, 5, 5, 8.0)
    results = []
    for tile in ((13, 8), (5, 8), (13, 4)):
        with RelativeSolver(A3, grid, local_precision="float32") as s:
            s.set_tile(*tile)
            s.initialize()
            s.advance(0.05)
            results.append((s.field().copy(), s.arrival().copy(), s.stats()[0]))
    for field, arrival, residual in results[1:]:
        np.testing.assert_array_equal(bits(field), bits(results[0][0]))
        np.testing.assert_array_equal(bits(arrival), bits(results[0][1]))
        assert residual == results[0][2]
