"""Reader of completed relative tables (the output contract of free_dp.solve).

Restates the query semantics of pursuit-evasion-core
src/pursuit_evasion/reversible/relative_table.py so that tables written by
this package (or by the reference) can be read without the reference:
    * metadata checks                      relative_table.py:14-61
    * 32-corner multilinear stencil with
      periodic heading, [x,y,psi,vP,vE] ->
      storage [vP,vE,psi,y,x]              relative_table.py:76-102
    * signed field at a budget             relative_table.py:104-117
    * capture time = first zero crossing
      by bisection over frames             relative_table.py:119-161
`DeviceRelativeTable` answers the same queries with the table on the GPU.
"""

from __future__ import annotations

from itertools import product
import json
from pathlib import Path

import numpy as np

from .free_dp import SCHEMA, physics_signature

_BITS = np.array(list(product([0, 1], repeat=5)), dtype=np.int64)


class RelativeTable:
    state_dimension = 5

    def __init__(self, folder, config=None, *, max_budget=None):
        self.folder = Path(folder).resolve()
        self.meta = json.loads((self.folder / "meta.json").read_text())
        if self.meta.get("schema") != SCHEMA:
            raise ValueError("Not a reversible relative5D table")
        if self.meta["status"] != "complete" or not self.meta["history_saved"]:
            raise ValueError("A completed solve with signed history is required")
        if self.meta["tube_projection"] != "min over every internal update":
            raise ValueError("Unsupported budget convention")
        all_times = np.asarray(self.meta["times"], dtype=float)
        self.axes = tuple(np.asarray(a, dtype=float) for a in self.meta["axes"])
        self.shape = tuple(len(a) for a in self.axes)
        if len(self.axes) != 5 or min(self.shape) < 2:
            raise ValueError("Expected five nondegenerate coordinate axes")
        self.spacings = np.array([a[1] - a[0] for a in self.axes])
        for a, h in zip(self.axes, self.spacings):
            if not np.isfinite(a).all() or h <= 0 or not np.allclose(np.diff(a), h):
                raise ValueError("Axes must be finite, increasing and uniformly spaced")
        if not (np.isclose(self.axes[2][0], -np.pi)
                and np.isclose(self.spacings[2] * self.shape[2], 2 * np.pi)):
            raise ValueError("Heading axis must be periodic without a repeated endpoint")
        if "shape" in self.meta and tuple(self.meta["shape"]) != self.shape:
            raise ValueError("Metadata shape differs from coordinate axes")
        if len(all_times) < 2 or np.any(np.diff(all_times) <= 0):
            raise ValueError("Invalid output times")
        keep = len(all_times)
        if max_budget is not None:
            hits = np.flatnonzero(np.isclose(all_times, max_budget, rtol=0, atol=1e-10))
            if not len(hits) or hits[0] == 0:
                raise ValueError("max_budget must be a positive retained output budget")
            keep = hits[0] + 1
        self.times = all_times[:keep].copy()
        expected = int(np.prod(self.shape)) * len(all_times) * 4
        if (self.folder / "fields.f32").stat().st_size != expected:
            raise ValueError("History byte length differs from metadata")
        fields = np.memmap(self.folder / "fields.f32", mode="r", dtype=np.float32,
                           shape=(len(all_times), *self.shape))
        self.fields = fields[:keep]
        self._flat = self.fields.reshape(keep, -1)
        self._strides = np.cumprod((1,) + self.shape[:0:-1])[::-1]
        self.physics = self.meta["physics"]
        self.horizon = float(self.times[-1])
        if config is not None:
            self.assert_compatible(config)

    def assert_compatible(self, config):
        if physics_signature(config) != self.physics:
            raise ValueError("The free-space table does not match the vehicle/capture model")

    def stencil(self, states):
        """Flat indices [n,32], weights [n,32], validity [n] and batch shape."""
        states = np.asarray(states, dtype=float)
        if states.ndim < 1 or states.shape[-1] != 5:
            raise ValueError("Relative states must end in [x,y,psi,vP,vE]")
        batch = states.shape[:-1]
        q = states.reshape(-1, 5)[:, [3, 4, 2, 1, 0]]
        valid = np.isfinite(q).all(1)
        q = np.where(np.isfinite(q), q, 0)
        index = np.zeros((len(q), 32), dtype=np.int64)
        weight = np.ones((len(q), 32))
        for k, (axis, h, n) in enumerate(zip(self.axes, self.spacings, self.shape)):
            if k == 2:
                f = ((q[:, k] + np.pi) % (2 * np.pi)) / h
                lower = np.floor(f).astype(np.int64) % n
                frac = f - np.floor(f)
            else:
                valid &= (q[:, k] >= axis[0] - 1e-10) & (q[:, k] <= axis[-1] + 1e-10)
                f = (np.clip(q[:, k], axis[0], axis[-1]) - axis[0]) / h
                lower = np.minimum(np.floor(f).astype(np.int64), n - 2)
                frac = f - lower
            corner = lower[:, None] + _BITS[None, :, k]
            if k == 2:
                corner %= n
            index += corner * self._strides[k]
            weight *= np.where(_BITS[None, :, k], frac[:, None], 1 - frac[:, None])
        return index, weight, valid, batch

    def field(self, states, budget):
        index, weight, valid, batch = self.stencil(states)
        tau = np.broadcast_to(np.asarray(budget, dtype=float), batch).reshape(-1)
        valid &= np.isfinite(tau) & (tau >= 0) & (tau <= self.horizon + 1e-10)
        if not valid.any():
            return np.full(batch, np.nan)
        tau = np.where(np.isfinite(tau), tau, 0)
        k = np.clip(np.searchsorted(self.times, tau, side="right") - 1, 0,
                    len(self.times) - 2)
        frac = (tau - self.times[k]) / (self.times[k + 1] - self.times[k])
        a = (self._flat[k[:, None], index] * weight).sum(1)
        b = (self._flat[(k + 1)[:, None], index] * weight).sum(1)
        return np.where(valid, a + frac * (b - a), np.nan).reshape(batch)

    def _physical(self, flat):
        ok = np.isfinite(flat).all(1)
        for k, role in ((3, "pursuer"), (4, "evader")):
            ok &= (flat[:, k] >= self.physics[role]["speed_min"] - 1e-10) & (
                flat[:, k] <= self.physics[role]["speed_max"] + 1e-10)
        return ok

    def value(self, states):
        """Capture time: first crossing of the interpolated signed fields."""
        index, weight, valid, batch = self.stencil(states)
        flat = np.asarray(states, dtype=float).reshape(-1, 5)
        captured = np.linalg.norm(flat[:, :2], axis=1) <= self.physics["capture_radius"]
        if not valid.any():
            return np.where(captured & self._physical(flat), 0.0, np.nan).reshape(batch)

        def sample(k):
            return (self._flat[np.asarray(k)[:, None], index] * weight).sum(1)

        lo = np.zeros(len(index), dtype=int)
        hi = np.full(len(index), len(self.times) - 1, dtype=int)
        valid &= sample(hi) <= 0
        while np.any(hi - lo > 1):
            mid = (lo + hi) // 2
            inside = sample(mid) <= 0
            hi = np.where(inside, mid, hi)
            lo = np.where(inside, lo, mid)
        a, b = sample(lo), sample(hi)
        frac = np.divide(a, a - b, out=np.zeros_like(a), where=abs(a - b) > 1e-14)
        out = self.times[lo] + np.clip(frac, 0, 1) * (self.times[hi] - self.times[lo])
        out = np.where(valid, out, np.nan)
        return np.where(captured & self._physical(flat), 0, out).reshape(batch)


class DeviceRelativeTable:
    """A completed table resident on a CUDA device (pe_table_*): the same
    `field` and `value` queries as RelativeTable, for batches of states,
    evaluated by GPU kernels in double precision."""

    def __init__(self, table, device=0):
        import ctypes

        from .. import _native

        self._ctypes = ctypes
        self._native = _native
        self._lib = _native.library()
        self.table = table
        frames = np.ascontiguousarray(table.fields, dtype=np.float32)
        times = np.ascontiguousarray(table.times, dtype=np.float64)
        shape = (ctypes.c_int32 * 5)(*table.shape)
        lo = (ctypes.c_double * 5)(*[float(a[0]) for a in table.axes])
        hi = (ctypes.c_double * 5)(*[float(a[-1]) for a in table.axes])
        h = (ctypes.c_double * 5)(*[float(x) for x in table.spacings])
        ph = table.physics
        limits = (ctypes.c_double * 4)(ph["pursuer"]["speed_min"], ph["pursuer"]["speed_max"],
                                       ph["evader"]["speed_min"], ph["evader"]["speed_max"])
        handle = ctypes.c_void_p()
        _native.check(self._lib.pe_table_create(
            frames.ctypes.data, len(times), times.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            shape, lo, hi, h, float(ph["capture_radius"]), limits, int(device),
            ctypes.byref(handle)))
        self._h = handle

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pe_table_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _states(self, states):
        states = np.asarray(states, dtype=np.float64)
        if states.ndim < 1 or states.shape[-1] != 5:
            raise ValueError("Relative states must end in [x,y,psi,vP,vE]")
        return np.ascontiguousarray(states.reshape(-1, 5)), states.shape[:-1]

    def value(self, states):
        flat, batch = self._states(states)
        out = np.empty(len(flat), np.float64)
        if len(flat):
            dp = self._ctypes.POINTER(self._ctypes.c_double)
            self._native.check(self._lib.pe_table_value(
                self._h, flat.ctypes.data_as(dp), len(flat), out.ctypes.data_as(dp)))
        return out.reshape(batch)

    def field(self, states, budget):
        flat, batch = self._states(states)
        tau = np.ascontiguousarray(
            np.broadcast_to(np.asarray(budget, dtype=np.float64), batch).reshape(-1))
        out = np.empty(len(flat), np.float64)
        if len(flat):
            dp = self._ctypes.POINTER(self._ctypes.c_double)
            self._native.check(self._lib.pe_table_field(
                self._h, flat.ctypes.data_as(dp), tau.ctypes.data_as(dp), len(flat),
                out.ctypes.data_as(dp)))
        return out.reshape(batch)
