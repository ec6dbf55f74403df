"""The FP64-table error statistics on CPU: the subsampled tile (every
`step`-th x, y and psi node from 0, every speed) and its error summary, and
the FP64-storage handle's option checks, which run before any device
work."""

import numpy as np
import pytest

from pursuit_evasion_b200.reversible.fp64_table import (
    RelativeSolverF64,
    subsample,
    subsampled_error,
)
from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
from tests.helpers import A3


def test_subsampled_tile_and_error_summary():
    grid = RelativeGrid(65, 48, 3, 3, 8.0)
    rng = np.random.default_rng(0)
    ref = rng.normal(size=grid.shape)
    tile = subsample(ref, 8)
    assert tile.shape == (3, 3, 6, 9, 9)  # x, y: 0..64 step 8; psi: 0..40
    np.testing.assert_array_equal(tile[1, 2, 3, 4, 5], ref[1, 2, 24, 32, 40])
    table = ref.astype(np.float32)
    table[0, 0, 8, 16, 24] += 1e-3  # on the tile
    table[0, 0, 9, 16, 24] += 1.0   # off the tile: not seen
    e = subsampled_error(table, ref, 8)
    assert e["nodes"] == 3 * 3 * 6 * 9 * 9 and e["step"] == 8
    assert e["max_abs"] == pytest.approx(1e-3, rel=1e-3)
    assert 0 < e["p999_abs"] < 1e-6 < e["max_abs"]  # one outlier in 13,122 nodes
    assert e["mean_abs"] < 5e-7  # float32 rounding of N(0, 1) values plus the outlier


def test_fp64_solver_rejects_invalid_options_before_device_work():
    with pytest.raises(ValueError):
        RelativeSolverF64(A3, RelativeGrid(17, 12, 7, 7, 4.0), order=3)
