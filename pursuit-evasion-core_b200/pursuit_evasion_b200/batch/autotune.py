"""Tile autotuner of the batched solver.

A work item of the exact batched kernel is `rows` y rows of one (vP, vE,
psi) plane of one solve; one of the tiled float32 kernel is `rows` y rows of
one (vP, vE) plane stack over all headings, a thread per 4-cell x chunk (at
most 256 / ceil(positions / 4) rows).  Fewer rows give more, smaller items
(better balance across the CTAs); more rows the reverse (less y halo per
cell), and the best choice depends on the grid width.  `tune` times every candidate row count on a few
solves of each width bucket (each solve cut to a short horizon, so a trial
is a few RK2 steps) and keeps the fastest; the winners are cached in a JSON
file keyed by device name and arithmetic, and `apply` sets them on a
`BatchSolver`.
"""

from __future__ import annotations

import json
import os
from dataclasses import replace
from pathlib import Path

from . import BatchSolver

BUCKETS = ((17, 24), (25, 32), (33, 40), (41, 49))
CANDIDATE_ROWS = (4, 8, 12, 16, 24, 32)


def bucket_of(positions):
    for lo, hi in BUCKETS:
        if lo <= positions <= hi:
            return f"{lo}-{hi}"
    return "other"


def default_cache():
    root = os.environ.get("PE_B200_CACHE") or os.path.join(
        os.environ.get("XDG_CACHE_HOME", os.path.expanduser("~/.cache")), "pe_b200")
    return Path(root) / "batch_tiles.json"


def _device_name(device):
    import torch

    return torch.cuda.get_device_name(device)


def candidates(narrowest, local_precision="float64", widest=None):
    """Row counts to try for a bucket whose grids have `narrowest` to
    `widest` positions: exact kernel, those that give every thread of a
    256-thread CTA a cell; tiled float32 kernel, those up to the capacity of
    a CTA on the widest grid (one 4-cell chunk per thread)."""
    if local_precision == "float32":
        widest = narrowest if widest is None else max(widest, narrowest)
        cap = min(narrowest, 256 // ((widest + 3) // 4))
        return sorted({min(r, cap) for r in CANDIDATE_ROWS if r <= narrowest} | {cap})
    rows = [r for r in CANDIDATE_ROWS if r <= narrowest and r * narrowest >= 256]
    return rows or [narrowest]


def tune(solves, *, device=0, local_precision="float32", per_bucket=6, trial_steps=4,
         repeats=2, cache=None, log=None):
    """Fastest rows per width bucket for these solves: {bucket: rows}."""
    import torch

    cache = Path(cache) if cache else default_cache()
    key = f"{_device_name(device)} {local_precision}" + (" tiled" if local_precision == "float32"
                                                         else "")
    try:
        table = json.loads(cache.read_text())
    except (OSError, ValueError):
        table = {}
    known = table.get(key, {})
    groups = {}
    for s in solves:
        groups.setdefault(bucket_of(s.grid.positions), []).append(s)
    result = {}
    for bucket, members in sorted(groups.items()):
        if bucket in known:
            result[bucket] = known[bucket]
            continue
        sample = members[:per_bucket]
        timings = {}
        with BatchSolver([replace(s, horizon=1.0) for s in sample], device=device) as probe:
            limits = [probe.info(i)["dt_limit"] for i in range(len(sample))]
        trial = [replace(s, horizon=trial_steps * lim) for s, lim in zip(sample, limits)]
        with BatchSolver(trial, local_precision=local_precision, device=device) as b:
            widths = [s.grid.positions for s in members]
            for rows in candidates(min(widths), local_precision, max(widths)):
                for i in range(len(trial)):
                    b.set_tile(i, rows)
                best = None
                for _ in range(repeats):
                    b.initialize()
                    b.profile(True)
                    b.run()
                    ms, _ = b.kernel_time()
                    b.profile(False)
                    b.synchronize()
                    best = ms if best is None else min(best, ms)
                timings[rows] = best
        torch.cuda.synchronize(device)
        winner = min(timings, key=timings.get)
        result[bucket] = winner
        if log:
            log(f"bucket {bucket}: " + ", ".join(f"{r} rows {t:.3f} ms"
                                                 for r, t in timings.items())
                + f" -> {winner}")
    table[key] = {**known, **result}
    try:
        cache.parent.mkdir(parents=True, exist_ok=True)
        cache.write_text(json.dumps(table, indent=1, sort_keys=True))
    except OSError:
        pass
    return result


def apply(batch, tiles):
    """Set each solve's tile from a {bucket: rows} table."""
    for i, s in enumerate(batch.solves):
        rows = tiles.get(bucket_of(s.grid.positions))
        if rows:
            batch.set_tile(i, min(int(rows), s.grid.positions))
