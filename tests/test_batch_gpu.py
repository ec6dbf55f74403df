"""Batched relative 5D solves in one persistent launch (pe_batch_*): every
solve of a heterogeneous batch equals, bit for bit, a float64
RelativeSolver advanced to the same horizon, and the oracle's restatement of
the reference executable; results do not depend on the work-item tile; the
float32 cell update tracks the exact one; the tile autotuner returns a row
count per width bucket."""

import numpy as np
import pytest

from pursuit_evasion_b200.batch import BatchSolve, BatchSolver, draw_batch
from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
from pursuit_evasion_b200.reversible.relative_solver import RelativeSolver
from tests.helpers import A3, CONFIG1_GRID, bits

pytestmark = pytest.mark.gpu


def small_batch():
    solves = draw_batch(7, count=5)
    # keep them small: shrink grids, keep the drawn physics and horizons
    out = []
    for k, s in enumerate(solves):
        g = s.grid
        grid = RelativeGrid(min(g.positions, 13 + 4 * k), min(g.headings, 12),
                            min(g.p_speeds, 7), min(g.e_speeds, 7), g.extent)
        out.append(BatchSolve(s.config, grid, min(s.horizon, 0.3 + 0.1 * k)))
    out.append(BatchSolve(A3, CONFIG1_GRID, 0.2))  # the README smoke grid
    return out


def test_every_solve_equals_the_single_grid_exact_path():
    solves = small_batch()
    with BatchSolver(solves) as b:
        b.initialize()
        b.run()
        b.synchronize()
        got = [(b.field(i).ravel().copy(), b.arrival(i).ravel().copy(), b.info(i))
               for i in range(len(solves))]
    for s, (field, arrival, info) in zip(solves, got):
        with RelativeSolver(s.config, s.grid, local_precision="float64") as r:
            r.initialize()
            steps = r.advance(s.horizon)
            ref_field, ref_arrival = r.field().ravel(), r.arrival().ravel()
        assert info["steps"] == steps
        np.testing.assert_array_equal(bits(field), bits(ref_field))
        np.testing.assert_array_equal(bits(arrival), bits(ref_arrival))


def test_batch_matches_the_oracle_reference_solve(oracle):
    """The README grid solved to 0.2 s inside a batch equals the oracle's
    restatement of native_relative.cpp (pinned to the reference executable
    by the golden vectors) with one frame at the horizon."""
    solves = small_batch()
    idx = len(solves) - 1
    with BatchSolver(solves) as b:
        b.initialize()
        b.run()
        field = b.field(idx).ravel()
        arrival = b.arrival(idx).ravel()
    cfg = oracle.rel_cfg(A3, CONFIG1_GRID)
    frames, ref_arrival, _ = oracle.rel_solve_f32(cfg, 0.2, 0.2)
    np.testing.assert_array_equal(bits(field), bits(frames[-1]))
    np.testing.assert_array_equal(bits(arrival), bits(ref_arrival))


def test_results_do_not_depend_on_the_tile():
    solves = small_batch()[:3]
    fields = []
    for rows in (1, 3):
        with BatchSolver(solves) as b:
            for i in range(len(solves)):
                b.set_tile(i, rows)
                assert b.tile(i) == rows
            b.initialize()
            b.run()
            fields.append([b.field(i).ravel().copy() for i in range(len(solves))])
    for a, c in zip(*fields):
        np.testing.assert_array_equal(bits(a), bits(c))


def test_rerun_after_init_repeats_the_solution():
    solves = small_batch()[:2]
    with BatchSolver(solves) as b:
        out = []
        for _ in range(2):
            b.initialize()
            b.run()
            out.append(b.field(1).ravel().copy())
        with pytest.raises(RuntimeError):
            b.run()  # the fields hold a solution: init first
    np.testing.assert_array_equal(bits(out[0]), bits(out[1]))


def test_float32_batch_tracks_the_exact_path(oracle):
    """The float32 cell update over whole solves (up to ~100 RK2 steps).  Each
    step rounds differently and now and then flips an ENO2 selection, and
    later steps carry that to the neighbouring cells, so the bound is the
    scheme's own float sensitivity: per solve, |float32 - exact| stays within
    twice |exact - FP64-storage oracle|, the gap between the reference's own
    float32 storage and double storage (max and mean), plus float rounding."""
    solves = small_batch()
    out = {}
    for precision in ("float64", "float32"):
        with BatchSolver(solves, local_precision=precision) as b:
            b.initialize()
            b.run()
            b.synchronize()
            out[precision] = [b.field(i).ravel().astype(np.float64)
                              for i in range(len(solves))]
    for s, fast, exact in zip(solves, out["float32"], out["float64"]):
        f64, _ = oracle.rel_solve_f64(oracle.rel_cfg(s.config, s.grid), s.horizon, s.horizon)
        storage = np.abs(exact - f64)
        diff = np.abs(fast - exact)
        assert diff.max() <= 2 * storage.max() + 2e-5, (diff.max(), storage.max())
        assert diff.mean() <= 2 * storage.mean() + 1e-6, (diff.mean(), storage.mean())


def test_autotuner_picks_a_tile_per_bucket(tmp_path):
    from pursuit_evasion_b200.batch import autotune

    solves = draw_batch(3, count=12)
    tiles = autotune.tune(solves, per_bucket=2, trial_steps=2, repeats=1,
                          cache=tmp_path / "tiles.json")
    assert set(tiles) == {autotune.bucket_of(s.grid.positions) for s in solves}
    for bucket, rows in tiles.items():
        widths = [s.grid.positions for s in solves
                  if autotune.bucket_of(s.grid.positions) == bucket]
        assert rows in autotune.candidates(min(widths), "float32", max(widths))
    assert (tmp_path / "tiles.json").exists()
    with BatchSolver(solves[:2], local_precision="float32") as b:
        autotune.apply(b, tiles)
        assert b.tile(0) == min(tiles[autotune.bucket_of(solves[0].grid.positions)],
                                solves[0].grid.positions)
