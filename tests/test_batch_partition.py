"""Splitting a batch of independent solves over several GPUs
(pursuit_evasion_b200.batch.partition): every solve lands on exactly one
rank, the shares are balanced within one solve's work, the split is the
same on every rank (checked on two gloo ranks), and the step count per solve
follows the batched solver's schedule (CFL steps, the last one cut to the
horizon)."""

import os

import pytest

from pursuit_evasion_b200.batch import (draw_batch, local_share, partition, solve_steps,
                                        solve_work)
from pursuit_evasion_b200.reversible.relative_solver import cfl_limit


def test_partition_covers_every_solve_once_and_balances():
    solves = draw_batch(0, 64)
    work = [solve_work(s) for s in solves]
    for parts in (1, 2, 3, 8):
        shares = partition(solves, parts)
        assert len(shares) == parts
        flat = sorted(i for sh in shares for i in sh)
        assert flat == list(range(len(solves)))
        loads = [sum(work[i] for i in sh) for sh in shares]
        assert max(loads) - min(loads) <= max(work)
    assert partition(solves, 1) == [list(range(len(solves)))]
    with pytest.raises(ValueError):
        partition(solves, 0)


def test_steps_follow_the_batch_schedule():
    for s in draw_batch(3, 8):
        limit = cfl_limit(s.config, s.grid)
        n = solve_steps(s)
        assert (n - 1) * limit < s.horizon <= n * limit + 1e-12


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        solves = draw_batch(1, 40)
        idx, mine = local_share(solves, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, (rank, idx, partition(solves, world)))
        out.put(gathered if rank == 0 else None)
    finally:
        dist.destroy_process_group()


def test_every_rank_computes_the_same_split():
    import multiprocessing as mp
    import socket

    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gathered = next(r for r in results if r is not None)
    (_, idx0, split0), (_, idx1, split1) = sorted(gathered)
    assert split0 == split1
    assert idx0 == split0[0] and idx1 == split0[1]
    assert sorted(idx0 + idx1) == list(range(40))
