"""Signed-front queries of a completed 6D square-game table.

The interface is the reference's reader (dp/table.py:17-123): a folder with
`meta.json` and `fields.f32` frames [T, xP, yP, thetaP, xE, yE, thetaE];
`stencil` (64-corner multilinear weights, periodic headings, positions
clamped to the box with out-of-box queries invalid), `field(states, budget)`
(the signed field, linear in time between frames) and `value(states)` (the
first budget at which the signed field reaches zero, NaN when unresolved,
0 for a capture or an evader fault at the state itself, NaN for a pursuer
outside the arena).  Capture times are not interpolated across jumps: the
signed field is sampled frame by frame and the crossing interpolated
between the last positive and the first non-positive frame.

The implementation is this package's: the corner set is built axis by axis
as an outer product of (lower, upper) node offsets and weights, and since
the stored fields are monotone non-increasing by budget (the declared
"min over every internal update" convention), the first non-positive frame
is found by sampling the frames in blocks of queries.  NumPy only; the
table may come from this package's solver or from the reference's.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from ..model import GameConfig
from .grid import GridSpec

_PERIODIC = (2, 5)
_CHUNK = 4096  # queries per block of frame samples


class LocalTable:
    def __init__(self, folder):
        self.folder = Path(folder)
        self.meta = json.loads((self.folder / "meta.json").read_text())
        if self.meta["status"] != "complete" or not self.meta["history_saved"]:
            raise ValueError("A completed solve with retained signed fields is required.")
        if self.meta.get("tube_projection") != \
                "min over every internal update, then max with avoid":
            raise ValueError(
                "This query requires the declared monotone-by-budget field convention.")
        spec = self.meta["grid"]
        self.grid = GridSpec(spec["positions"], spec["headings"], spec["extent"])
        self.config = GameConfig.from_dict(self.meta["config"])
        self.times = np.array(self.meta["times"])
        path = self.folder / "fields.f32"
        frames = len(self.times)
        self.fields = np.memmap(path, dtype=np.float32, mode="r",
                                shape=(frames, *self.grid.shape))
        if self.fields.nbytes != path.stat().st_size:
            raise ValueError("Field length does not match metadata.")
        self._frames = self.fields.reshape(frames, -1)
        shape = self.grid.shape
        # element stride of each axis in a C-ordered frame
        self._stride = [int(np.prod(shape[k + 1:])) for k in range(6)]

    # ------------------------------------------------------------ stencil
    def _bracket(self, k, q, valid):
        """Lower node and upper weight of coordinate q on axis k."""
        n = self.grid.shape[k]
        h = self.grid.spacings[k]
        if k in _PERIODIC:
            f = np.mod(q + np.pi, 2 * np.pi) / h
            base = np.floor(f)
            return base.astype(np.int64) % n, f - base, valid
        axis = self.grid.axes[k]
        lo_edge, hi_edge = axis[0], axis[-1]
        valid = valid & (q >= lo_edge - 1e-10) & (q <= hi_edge + 1e-10)
        f = (np.clip(q, lo_edge, hi_edge) - lo_edge) / h
        node = np.minimum(np.floor(f).astype(np.int64), n - 2)
        return node, f - node, valid

    def stencil(self, states):
        """64-corner multilinear stencil of states [..., 6] = [xP, yP, thetaP,
        xE, yE, thetaE]: flat indices [N, 64], weights [N, 64], validity [N]
        and the batch shape."""
        states = np.asarray(states, dtype=float)
        if states.shape[-1] != 6:
            raise ValueError("State order must be [xP,yP,thetaP,xE,yE,thetaE].")
        batch = states.shape[:-1]
        s = states.reshape(-1, 6)
        finite = np.isfinite(s)
        valid = finite.all(axis=1)
        s = np.where(finite, s, 0.0)
        index = np.zeros((len(s), 1), np.int64)
        weight = np.ones((len(s), 1))
        for k in range(6):
            node, w, valid = self._bracket(k, s[:, k], valid)
            upper = node + 1
            if k in _PERIODIC:
                upper %= self.grid.shape[k]
            # the two nodes of this axis, as flat offsets and weights
            off = np.stack([node, upper], axis=1) * self._stride[k]
            wk = np.stack([1.0 - w, w], axis=1)
            index = (index[:, :, None] + off[:, None, :]).reshape(len(s), -1)
            weight = (weight[:, :, None] * wk[:, None, :]).reshape(len(s), -1)
        return index, weight, valid, batch

    def _sample(self, frame, index, weight):
        """Signed field at frame index/indices `frame` (scalar or [N])."""
        rows = self._frames[np.asarray(frame)[..., None], index] if np.ndim(frame) else \
            self._frames[int(frame)][index]
        return np.einsum("nc,nc->n", rows, weight)

    # ------------------------------------------------------------ queries
    def field(self, states, budget):
        """Signed field at `budget` (linear in time between frames)."""
        index, weight, valid, batch = self.stencil(states)
        tau = np.broadcast_to(np.asarray(budget, dtype=float), batch).reshape(-1)
        valid &= np.isfinite(tau) & (tau >= 0) & (tau <= self.times[-1] + 1e-10)
        last = len(self.times) - 2
        k = np.clip(np.searchsorted(self.times, tau, side="right") - 1, 0, last)
        span = self.times[k + 1] - self.times[k]
        before = self._sample(k, index, weight)
        after = self._sample(k + 1, index, weight)
        out = before + (after - before) * ((tau - self.times[k]) / span)
        return np.where(valid, out, np.nan).reshape(batch)

    def _first_crossing(self, index, weight):
        """Per query: the first frame whose sample is <= 0 (len(times) when
        none is), from frame samples taken in blocks of queries."""
        frames = len(self.times)
        first = np.full(len(index), frames, np.int64)
        for start in range(0, len(index), _CHUNK):
            sl = slice(start, start + _CHUNK)
            samples = np.stack([self._sample(f, index[sl], weight[sl])
                                for f in range(frames)], axis=1)
            inside = samples <= 0
            hit = inside.any(axis=1)
            first[sl] = np.where(hit, inside.argmax(axis=1), frames)
        return first

    def value(self, states):
        """First numerical success time; NaN means unresolved or invalid, not
        escape.  Capture and evader faults at the state itself give 0, a
        pursuer outside the arena NaN."""
        index, weight, valid, batch = self.stencil(states)
        frames = len(self.times)
        first = self._first_crossing(index, weight)
        valid &= first < frames                    # reaches zero within the table
        hi = np.clip(first, 1, frames - 1)         # first non-positive frame
        lo = hi - 1                                # last positive one (or frame 0)
        a = self._sample(lo, index, weight)
        b = self._sample(hi, index, weight)
        drop = a - b
        frac = np.zeros_like(a)
        np.divide(a, drop, out=frac, where=np.abs(drop) > 1e-14)
        when = self.times[lo] + np.clip(frac, 0.0, 1.0) * (self.times[hi] - self.times[lo])

        s = np.asarray(states, dtype=float).reshape(-1, 6)
        c = self.config
        pursuer_in = np.abs(s[:, :2]).max(axis=1) < c.arena_half_width
        captured = np.hypot(s[:, 0] - s[:, 3], s[:, 1] - s[:, 4]) <= c.capture_radius
        evader_out = np.abs(s[:, 3:5]).max(axis=1) >= c.arena_half_width
        result = np.where(valid & pursuer_in, when, np.nan)
        immediate = np.isfinite(s).all(axis=1) & pursuer_in & (captured | evader_out)
        return np.where(immediate, 0.0, result).reshape(batch)
