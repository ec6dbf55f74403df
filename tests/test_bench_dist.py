"""The replica bench's multi-rank host logic on CPU ranks (gloo, world size
2): environment parsing, the max-over-ranks timing reduction every rank
takes, and the reference arm's rank-0-only rule."""

import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

REPO = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, str(REPO))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime

    import bench

    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r reports (r + 1, 10 - r): every rank gets the maxima
        got = bench.max_over_ranks([rank + 1.0, 10.0 - rank], world, device="cpu")
        # the reference arm prints on rank 0 only; other ranks return at once
        printed = bench.run_reference_arm(None, world, rank) if rank else "rank0"
        out.put((rank, got, printed))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rank_zero_rule():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    results = sorted(out.get(timeout=10) for _ in procs)
    assert results[0][1] == [2.0, 10.0] and results[1][1] == [2.0, 10.0]
    assert results[1][2] is None  # rank 1 did no reference work


def _sharded_rank(rank, world, port, out):
    sys.path.insert(0, str(REPO))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from types import SimpleNamespace

    import bench
    from tests import oracle_lib
    from tests.helpers import A3, CONFIG1_GRID
    from tests.shard_oracle import OracleShard

    bench.HORIZON = 0.2  # two 0.1-s frames of the README grid
    oracle = oracle_lib.load()
    try:
        line = bench.run_sharded(
            SimpleNamespace(steps=2, warmup=1, precision="float64"), world, rank, 0,
            backend="gloo", grid=CONFIG1_GRID,
            shard_factory=lambda b, e: OracleShard(oracle, A3, CONFIG1_GRID, b, e))
        out.put((rank, line))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_bench_on_gloo_ranks():
    """`bench.py --gpus N` (sharded mode) drives one table over N ranks:
    every rank takes the same steps and collectives, rank 0 prints a strong
    scaling line over the whole table with its vP ranges and copy bytes."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert results[1] is None
    line = results[0]
    assert line["scaling"] == "strong" and line["n_gpus"] == 2
    assert line["run"]["vp_ranges"] == [[0, 4], [4, 7]]
    assert line["value"] > 0 and line["e2e"]["value"] > 0
    slab = 12 * 17 * 17 * 7
    assert line["e2e"]["h2d_bytes_per_step"] == 4 * slab * (6 + 5)
    assert line["e2e"]["d2h_bytes_per_step"] == 8 * slab * 7
