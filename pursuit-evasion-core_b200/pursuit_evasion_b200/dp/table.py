"""Portable signed-front queries of a completed 6D square-game solve
(src/pursuit_evasion/dp/table.py:17-123).  Capture times are not
interpolated across jumps: the signed field is interpolated at each budget
and its first zero crossing located by bisection over the frames.  NumPy
only; the table may come from this package's solver or the reference's."""

from __future__ import annotations

from itertools import product
import json
from pathlib import Path

import numpy as np

from ..model import GameConfig
from .grid import GridSpec

PERIODIC = (2, 5)


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
        g = self.meta["grid"]
        self.grid = GridSpec(g["positions"], g["headings"], g["extent"])
        self.config = GameConfig.from_dict(self.meta["config"])
        self.times = np.array(self.meta["times"])
        self.fields = np.memmap(self.folder / "fields.f32", dtype=np.float32, mode="r",
                                shape=(len(self.times), *self.grid.shape))
        if self.fields.nbytes != (self.folder / "fields.f32").stat().st_size:
            raise ValueError("Field length does not match metadata.")
        self._flat = self.fields.reshape(len(self.times), -1)
        self._strides = np.cumprod((1,) + self.grid.shape[:0:-1])[::-1]
        self._corners = np.array(list(product([0, 1], repeat=6)), dtype=np.int64)

    def stencil(self, states):
        """64-corner multilinear stencil (flat indices, weights), validity and
        the batch shape of states [..., 6] = [xP, yP, thetaP, xE, yE, thetaE]."""
        states = np.asarray(states, dtype=float)
        if states.shape[-1] != 6:
            raise ValueError("State order must be [xP,yP,thetaP,xE,yE,thetaE].")
        shape = states.shape[:-1]
        s = states.reshape(-1, 6)
        valid = np.isfinite(s).all(1)
        s = np.where(np.isfinite(s), s, 0.0)
        lower, frac = [], []
        for k, (axis, n, h) in enumerate(zip(self.grid.axes, self.grid.shape,
                                             self.grid.spacings)):
            q = s[:, k]
            if k in PERIODIC:
                f = ((q + np.pi) % (2 * np.pi)) / h
                j = np.floor(f).astype(int) % n
                w = f - np.floor(f)
            else:
                valid &= (q >= axis[0] - 1e-10) & (q <= axis[-1] + 1e-10)
                f = (np.clip(q, axis[0], axis[-1]) - axis[0]) / h
                j = np.minimum(np.floor(f).astype(int), n - 2)
                w = f - j
            lower.append(j)
            frac.append(w)
        index = np.zeros((len(s), 64), np.int64)
        weight = np.ones((len(s), 64))
        for k, (j, w, n) in enumerate(zip(lower, frac, self.grid.shape)):
            coord = j[:, None] + self._corners[None, :, k]
            if k in PERIODIC:
                coord %= n
            index += coord * self._strides[k]
            weight *= np.where(self._corners[None, :, k], w[:, None], 1 - w[:, None])
        return index, weight, valid, shape

    def field(self, states, budget):
        """Signed field at `budget` (linear in time between frames)."""
        index, weight, valid, shape = self.stencil(states)
        tau = np.broadcast_to(np.asarray(budget), shape).reshape(-1)
        valid &= np.isfinite(tau) & (tau >= 0) & (tau <= self.times[-1] + 1e-10)
        k = np.clip(np.searchsorted(self.times, tau, side="right") - 1, 0, len(self.times) - 2)
        ratio = (tau - self.times[k]) / (self.times[k + 1] - self.times[k])
        a = (self._flat[k[:, None], index] * weight).sum(1)
        b = (self._flat[(k + 1)[:, None], index] * weight).sum(1)
        return np.where(valid, a + (b - a) * ratio, np.nan).reshape(shape)

    def value(self, states):
        """First numerical success time; NaN means unresolved or invalid, not
        escape.  Capture and evader faults at the state itself give 0, a
        pursuer outside the arena NaN."""
        index, weight, valid, shape = self.stencil(states)

        def sample(k):
            return (self._flat[np.asarray(k)[:, None], index] * weight).sum(1)

        lo = np.zeros(len(index), int)
        hi = np.full(len(index), len(self.times) - 1, int)
        valid &= sample(hi) <= 0
        while np.any(hi - lo > 1):
            mid = (hi + lo) // 2
            inside = sample(mid) <= 0
            hi = np.where(inside, mid, hi)
            lo = np.where(inside, lo, mid)
        a, b = sample(lo), sample(hi)
        fraction = np.divide(a, a - b, out=np.zeros_like(a), where=abs(a - b) > 1e-14)
        result = self.times[lo] + np.clip(fraction, 0, 1) * (self.times[hi] - self.times[lo])
        s = np.asarray(states).reshape(-1, 6)
        c = self.config
        p_valid = np.max(abs(s[:, :2]), axis=1) < c.arena_half_width
        capture = np.linalg.norm(s[:, :2] - s[:, 3:5], axis=1) <= c.capture_radius
        e_fault = np.max(abs(s[:, 3:5]), axis=1) >= c.arena_half_width
        result = np.where(valid & p_valid, result, np.nan)
        finite_state = np.isfinite(s).all(axis=1)
        result = np.where(finite_state & p_valid & (capture | e_fault), 0.0, result)
        return result.reshape(shape)
