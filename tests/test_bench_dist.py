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
