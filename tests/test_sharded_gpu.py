"""vP-slab shards on the GPU (pe_relative_shard_*): several shards of one
grid held by this process on cuda:0, their halos refreshed by device copies
after every stage, against the single-grid solve of the same precision
(exact and float32 kernels) and the oracle, bit for bit.  (Every GPU run here has one GPU: the NCCL exchange between ranks
is covered by the gloo tests of the same driver.)"""

import numpy as np
import pytest

from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
from pursuit_evasion_b200.reversible.relative_solver import RelativeSolver
from pursuit_evasion_b200.reversible.sharded import (
    LocalExchange,
    RelativeShard,
    ShardedSolver,
    partition,
)
from tests.helpers import A3, CONFIG1_GRID, bits

pytestmark = pytest.mark.gpu


def sharded_frames(grid, parts, order, goals, precision="float64"):
    shards = [RelativeShard(A3, grid, b, e, order=order, local_precision=precision)
              for b, e in partition(grid.p_speeds, parts, order)]
    try:
        for s in shards:
            s.initialize()
        solver = ShardedSolver(shards, LocalExchange(shards))
        frames = []
        for goal in goals:
            solver.advance(goal)
            frames.append(np.concatenate([s.field() for s in shards]))
        arrival = np.concatenate([s.arrival() for s in shards])
        return np.array(frames), arrival, solver.steps, solver.residual()
    finally:
        for s in shards:
            s.close()


def single_frames(grid, order, goals, precision="float64"):
    with RelativeSolver(A3, grid, order=order, local_precision=precision) as s:
        s.initialize()
        frames = []
        for goal in goals:
            s.advance(goal)
            frames.append(s.field().ravel().copy())
        return np.array(frames), s.arrival().ravel().copy(), s.steps, s.stats()[0]


@pytest.mark.parametrize("precision", ["float64", "float32"])
@pytest.mark.parametrize("grid, parts, order", [
    (CONFIG1_GRID, 2, 2), (CONFIG1_GRID, 3, 2), (CONFIG1_GRID, 7, 1),
    (RelativeGrid(33, 16, 9, 5, 4.0), 4, 2)])
def test_shards_equal_single_grid_solve(grid, parts, order, precision):
    goals = (0.1, 0.2, 0.3)
    got, arrival, steps, residual = sharded_frames(grid, parts, order, goals, precision)
    ref, ref_arrival, ref_steps, ref_residual = single_frames(grid, order, goals, precision)
    assert steps == ref_steps
    np.testing.assert_array_equal(bits(got), bits(ref))
    np.testing.assert_array_equal(bits(arrival), bits(ref_arrival))
    assert residual == ref_residual


def test_shards_equal_oracle(oracle):
    cfg = oracle.rel_cfg(A3, CONFIG1_GRID, order=2)
    frames, arrival, steps = oracle.rel_solve_f32(cfg, 0.2, 0.1)
    got, got_arrival, got_steps, _ = sharded_frames(CONFIG1_GRID, 3, 2, (0.1, 0.2))
    assert got_steps == steps
    np.testing.assert_array_equal(bits(got), bits(frames[1:]))
    np.testing.assert_array_equal(bits(got_arrival), bits(arrival))



def test_sharded_table_with_one_nccl_rank_equals_free_dp_solve(tmp_path):
    import socket

    import torch.distributed as dist

    from pursuit_evasion_b200.reversible import sharded
    from pursuit_evasion_b200.reversible.free_dp import solve

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                            world_size=1)
    try:
        meta = sharded.solve(A3, CONFIG1_GRID, tmp_path / "shards", horizon=0.2,
                             output_dt=0.1)
    finally:
        dist.destroy_process_group()
    solve(A3, CONFIG1_GRID, tmp_path / "single", horizon=0.2, output_dt=0.1)
    assert meta["vp_shards"] == [[0, 7]]
    for name in ("fields.f32", "final.f32", "arrival.f32"):
        np.testing.assert_array_equal(
            bits(np.fromfile(tmp_path / "shards" / name, np.float32)),
            bits(np.fromfile(tmp_path / "single" / name, np.float32)))
