"""vP-slab sharding of the relative solve on CPU: the partition and halo
plan, and the sharding driver with its two halo exchanges (in-process
copies; torch.distributed P2P over gloo ranks, world sizes 2 and 3) around
the oracle stage, against the unsharded oracle solve bit for bit."""

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from pursuit_evasion_b200.reversible.sharded import (
    DistExchange,
    LocalExchange,
    ShardedSolver,
    halo_plan,
    partition,
)
from tests.helpers import A3, CONFIG1_GRID, bits
from tests.shard_oracle import OracleShard

REPO = Path(__file__).resolve().parents[1]


def test_partition_and_halo_plan():
    assert partition(7, 3) == [(0, 3), (3, 5), (5, 7)]
    assert partition(21, 8) == [(0, 3), (3, 6), (6, 9), (9, 12), (12, 15), (15, 17),
                                (17, 19), (19, 21)]
    assert partition(5, 1) == [(0, 5)]
    with pytest.raises(ValueError):
        partition(5, 3, order=2)
    assert partition(5, 3, order=1) == [(0, 2), (2, 4), (4, 5)]
    # middle shard of 7 slabs in 3: owns 3-4, buffer 1-6
    plan = halo_plan((1, 7, 3, 5), 2, 7)
    assert plan == {"lower": ((3, 5), (1, 3)), "upper": ((3, 5), (5, 7))}
    assert halo_plan((0, 5, 0, 3), 2, 7) == {"upper": ((1, 3), (3, 5))}
    assert halo_plan((0, 7, 0, 7), 2, 7) == {}


def reference(oracle, order, horizon=0.2, output_dt=0.1):
    cfg = oracle.rel_cfg(A3, CONFIG1_GRID, order=order)
    return oracle.rel_solve_f32(cfg, horizon, output_dt)


@pytest.mark.parametrize("order, parts", [(2, 2), (2, 3), (1, 4)])
def test_local_exchange_equals_unsharded_oracle(oracle, order, parts):
    frames, arrival, steps = reference(oracle, order)
    shards = [OracleShard(oracle, A3, CONFIG1_GRID, b, e, order=order)
              for b, e in partition(CONFIG1_GRID.p_speeds, parts, order)]
    for s in shards:
        s.initialize()
    solver = ShardedSolver(shards, LocalExchange(shards))
    for k, goal in enumerate((0.1, 0.2), start=1):
        solver.advance(goal)
        got = np.concatenate([s.field() for s in shards])
        np.testing.assert_array_equal(bits(got), bits(frames[k]))
    assert solver.steps == steps
    np.testing.assert_array_equal(bits(np.concatenate([s.arrival() for s in shards])),
                                  bits(arrival))
    assert solver.residual() == max(s.stats()[0] for s in shards) > 0


def test_missing_exchange_is_detected(oracle):
    """Without the halo refresh the owned values differ: the check above
    would catch a wrong or missing exchange."""
    frames, _, _ = reference(oracle, 2)
    shards = [OracleShard(oracle, A3, CONFIG1_GRID, b, e)
              for b, e in partition(CONFIG1_GRID.p_speeds, 2)]
    for s in shards:
        s.initialize()
    solver = ShardedSolver(shards, lambda: None)
    solver.advance(0.1)
    got = np.concatenate([s.field() for s in shards])
    assert not np.array_equal(bits(got), bits(frames[1]))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, str(REPO))
    import datetime

    import torch.distributed as dist

    from tests import oracle_lib

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        oracle = oracle_lib.load()
        begin, end = partition(CONFIG1_GRID.p_speeds, world)[rank]
        shard = OracleShard(oracle, A3, CONFIG1_GRID, begin, end)
        shard.initialize()
        solver = ShardedSolver([shard], DistExchange(shard))
        fields = []
        for goal in (0.1, 0.2):
            solver.advance(goal)
            fields.append(shard.field())
        residual = solver.residual()
        out.put((rank, fields, shard.arrival(), solver.steps, residual, shard.stats()[0]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_dist_exchange_on_gloo_ranks_equals_unsharded_oracle(oracle, world):
    import torch.multiprocessing as mp

    frames, arrival, steps = reference(oracle, 2)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted((out.get(timeout=180) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for k in range(2):
        got = np.concatenate([r[1][k] for r in results])
        np.testing.assert_array_equal(bits(got), bits(frames[k + 1]))
    np.testing.assert_array_equal(bits(np.concatenate([r[2] for r in results])), bits(arrival))
    assert all(r[3] == steps for r in results)
    # every rank gets the maximum residual over ranks
    assert all(r[4] == max(q[5] for q in results) for r in results)


def test_shard_argument_errors_before_any_device_work():
    from pursuit_evasion_b200.reversible.sharded import RelativeShard

    with pytest.raises(ValueError, match="at least"):
        RelativeShard(A3, CONFIG1_GRID, 0, 1)  # one slab with a neighbour, order 2
    with pytest.raises(ValueError, match="begin < end"):
        RelativeShard(A3, CONFIG1_GRID, 3, 9)


def _table_rank(rank, world, port, folder, out):
    sys.path.insert(0, str(REPO))
    import datetime

    import torch.distributed as dist

    from pursuit_evasion_b200.reversible import sharded
    from tests import oracle_lib

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        oracle = oracle_lib.load()
        meta = sharded.solve(A3, CONFIG1_GRID, folder, horizon=0.2, output_dt=0.1,
                             shard_factory=lambda b, e: OracleShard(oracle, A3, CONFIG1_GRID,
                                                                    b, e))
        out.put((rank, meta["internal_steps"], meta["vp_shards"]))
    finally:
        dist.destroy_process_group()


def test_sharded_table_on_gloo_ranks_equals_oracle_and_reads_as_a_table(oracle, tmp_path):
    import torch.multiprocessing as mp

    from pursuit_evasion_b200.reversible.relative_table import RelativeTable

    frames, arrival, steps = reference(oracle, 2)
    folder = tmp_path / "table"
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_table_rank, args=(r, 2, port, str(folder), out))
             for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert all(r[1] == steps for r in results)
    assert results[0][2] == [[0, 4], [4, 7]]
    got = np.fromfile(folder / "fields.f32", np.float32).reshape(frames.shape)
    np.testing.assert_array_equal(bits(got), bits(frames))
    np.testing.assert_array_equal(bits(np.fromfile(folder / "final.f32", np.float32)),
                                  bits(frames[-1]))
    np.testing.assert_array_equal(bits(np.fromfile(folder / "arrival.f32", np.float32)),
                                  bits(arrival))
    table = RelativeTable(folder)
    assert table.shape == tuple(CONFIG1_GRID.shape)


def _refuse_rank(rank, world, port, folder, out):
    sys.path.insert(0, str(REPO))
    import datetime

    import torch.distributed as dist

    from pursuit_evasion_b200.reversible import sharded
    from tests import oracle_lib

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        oracle = oracle_lib.load()
        try:
            sharded.solve(A3, CONFIG1_GRID, folder, horizon=0.1, output_dt=0.1,
                          shard_factory=lambda b, e: OracleShard(oracle, A3, CONFIG1_GRID,
                                                                 b, e))
            out.put((rank, "solved"))
        except (FileExistsError, RuntimeError) as exc:
            out.put((rank, type(exc).__name__))
    finally:
        dist.destroy_process_group()


def test_sharded_table_refuses_existing_output_on_every_rank(tmp_path):
    """Rank 0 finds a non-empty folder; every rank stops before any work."""
    import torch.multiprocessing as mp

    folder = tmp_path / "table"
    folder.mkdir()
    (folder / "keep.txt").write_text("x")
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_refuse_rank, args=(r, 2, port, str(folder), out))
             for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert results == [(0, "FileExistsError"), (1, "RuntimeError")]
    assert sorted(x.name for x in folder.iterdir()) == ["keep.txt"]


def _failing_rank(rank, world, port, folder, out):
    sys.path.insert(0, str(REPO))
    import datetime

    import torch.distributed as dist

    from pursuit_evasion_b200.reversible import sharded
    from tests import oracle_lib

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        oracle = oracle_lib.load()

        def factory(b, e):
            if rank == 1:  # as pe_relative_shard_create failing on one GPU
                raise MemoryError("shard buffers do not fit")
            return OracleShard(oracle, A3, CONFIG1_GRID, b, e)

        try:
            sharded.solve(A3, CONFIG1_GRID, folder, horizon=0.2, output_dt=0.1,
                          shard_factory=factory)
            out.put((rank, "solved", ""))
        except (MemoryError, RuntimeError) as exc:
            out.put((rank, type(exc).__name__, str(exc)))
    finally:
        dist.destroy_process_group()


def test_shard_failure_on_one_rank_stops_every_rank(tmp_path):
    """The shard factory fails on rank 1 only: rank 1 raises its own error,
    rank 0 learns of it at the set-up agreement and raises too, and both
    leave before any halo exchange (no rank waits for a peer that left)."""
    import time

    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_rank, args=(r, 2, port, str(tmp_path / "t"), out))
             for r in range(2)]
    t0 = time.monotonic()
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert time.monotonic() - t0 < 50  # well inside the 60 s group timeout
    assert results[0][:2] == (0, "RuntimeError")
    assert "rank 1 failed during shard set-up" in results[0][2]
    assert results[1][:2] == (1, "MemoryError")
