"""Learned warm start: a surrogate trained by the package's own kernels on a
minimum-time table warm-starts value iteration, which converges to the same
table as the cold start (the plain DP decides the answer) in fewer
iterations; online queries of arbitrary states agree with the table."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_warm_start_converges_to_the_plain_table_faster():
    from pursuit_evasion_b200.learned.warm_start import time_to_converged
    from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
    from tests.helpers import A3

    grid = RelativeGrid(17, 12, 7, 7, 4.0)
    result, _ = time_to_converged(A3, grid, dt=0.05, tol=1e-5, samples=1 << 17,
                                  epochs=8, batch=4096,
                                  coarse_grid=RelativeGrid(9, 8, 7, 7, 4.0))
    plain, warm = result["plain"], result["warm_same_table"]
    assert plain["converged"] and warm["converged"]
    # both runs stop within the contraction bound of the same fixed point:
    # |u_k - u*| <= r_k * b / (1 - b), b = exp(-dt), r_k < tol
    bound = 2 * 1e-5 * np.exp(-0.05) / (1 - np.exp(-0.05))
    assert warm["max_abs_diff_vs_plain"] <= bound
    assert warm["iterations"] < plain["iterations"]
    # the minimum-time value has near-discontinuities (escape barriers) that a
    # small network smooths over: the mean error is small, the max is not
    assert warm["surrogate_mean_abs_error"] < 0.05
    coarse = result["warm_coarse_table"]
    assert coarse["converged"] and coarse["max_abs_diff_vs_plain"] <= bound


def test_query_batch_matches_table_at_nodes():
    from pursuit_evasion_b200.learned.mlp import ValueMLP
    from pursuit_evasion_b200.learned.train import (
        RelativeNodeSampler,
        predict_nodes,
        predict_states,
        train,
    )
    from pursuit_evasion_b200.learned.warm_start import converge
    from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
    from tests.helpers import A3

    grid = RelativeGrid(17, 12, 7, 7, 4.0)
    u, info = converge(A3, grid, dt=0.05, tol=1e-5)
    net = ValueMLP(6, seed=1, max_batch=4096)
    train(net, RelativeNodeSampler(A3, grid, u), samples=1 << 17, epochs=6, batch=4096)
    dev = u.device
    rng = np.random.default_rng(0)
    cells = rng.choice(grid.states, size=4096, replace=False)
    axes = grid.axes(A3)
    iv, ie, ip, iy, ix = np.unravel_index(cells, grid.shape)
    states = np.stack([axes[4][ix], axes[3][iy], axes[2][ip], axes[0][iv], axes[1][ie]], 1)
    q = predict_states(net, A3, grid.extent, torch.tensor(states, dtype=torch.float32,
                                                          device=dev))
    full = predict_nodes(net, RelativeNodeSampler(A3, grid), torch.empty(grid.states, device=dev))
    torch.testing.assert_close(q, full[torch.tensor(cells, device=dev)], rtol=0, atol=2e-2)
    err = (full - u).abs()
    assert float(err.mean()) < 0.05
