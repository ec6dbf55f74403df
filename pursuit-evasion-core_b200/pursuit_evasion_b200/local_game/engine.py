"""Vehicle geometry queries of the compact contact game on the GPU.

`GeometryEngine` has the interface of the reference's local_game/native.py
GeometryEngine (:135-230: `clearance`, `backup_safe`, `connections`,
`actions`) for one car of a `CircleArena`, answered by the
pe_geometry_* kernels of csrc/vehicle_geometry_exact.cu (one thread per
query) instead of an OpenMP library compiled at run time.  A car's model is
its limits, its rectangle in the arena and the control period.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .. import _native


class GeometryEngine:
    def __init__(self, arena, limits, role, threads=None, control_dt=0.05, device=0):
        self.arena = arena
        self.limits = limits
        self.role = role
        self.device = int(device)
        body = getattr(arena, role)
        self.model = _native.VehicleModel(
            speed_min=float(limits.speed_min), speed_max=float(limits.speed_max),
            acceleration=float(limits.acceleration),
            max_curvature=float(limits.max_curvature), length=float(body.length),
            width=float(body.width), control_dt=float(control_dt))
        self.obstacles = np.ascontiguousarray(arena.circles, np.float64).reshape(-1, 3)
        self._lib = _native.library()

    @staticmethod
    def _states(s):
        s = np.asarray(s, float)
        if s.shape[-1] != 4 or not np.isfinite(s).all():
            raise ValueError("Finite vehicle states[...,4] required")
        return np.ascontiguousarray(s.reshape(-1, 4))

    def _common(self):
        return (ctypes.c_void_p(self.obstacles.ctypes.data), len(self.obstacles),
                float(self.arena.half_width))

    def clearance(self, s):
        """Signed separation of the car's rectangle from walls and circles."""
        x = self._states(s)
        out = np.empty(len(x))
        _native.check(self._lib.pe_geometry_clearance(
            ctypes.byref(self.model), x.ctypes.data, len(x), *self._common(),
            out.ctypes.data, self.device))
        return out.reshape(np.shape(s)[:-1])

    def backup_safe(self, s):
        """Clear now, and one full-braking arc to rest is clear."""
        x = self._states(s)
        out = np.empty(len(x), np.uint8)
        _native.check(self._lib.pe_geometry_backup_safe(
            ctypes.byref(self.model), x.ctypes.data, len(x), *self._common(),
            out.ctypes.data, self.device))
        return out.astype(bool).reshape(np.shape(s)[:-1])

    def connections(self, start, target):
        """Straight configuration paths start[i] -> target[i] that stay clear."""
        a, b = self._states(start), self._states(target)
        if a.shape != b.shape:
            raise ValueError("Matched configuration arrays required")
        out = np.empty(len(a), np.uint8)
        _native.check(self._lib.pe_geometry_connections(
            ctypes.byref(self.model), a.ctypes.data, b.ctypes.data, len(a), *self._common(),
            out.ctypes.data, self.device))
        return out.astype(bool)

    def actions(self, s, controls, dt):
        """(ok [n, na], next [n, na, 4]): the held-control arc of every
        control over dt, ok where it is clear and ends backup safe."""
        x = self._states(s)
        u = np.ascontiguousarray(controls, float).reshape(-1, 2)
        ok = np.empty((len(x), len(u)), np.uint8)
        nxt = np.empty((len(x), len(u), 4))
        obstacles, n_obstacles, half = self._common()
        _native.check(self._lib.pe_geometry_actions(
            ctypes.byref(self.model), x.ctypes.data, len(x), u.ctypes.data, len(u),
            float(dt), obstacles, n_obstacles, half, ok.ctypes.data, nxt.ctypes.data,
            self.device))
        return ok.astype(bool), nxt
