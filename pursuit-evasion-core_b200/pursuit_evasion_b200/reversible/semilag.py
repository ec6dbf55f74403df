"""Semi-Lagrangian min-max backup of the relative 5D game (pe_semilag_*).

For every relative cell (x, y, psi, vP, vE) a backup takes the minimum over
the pursuer's 9 held actions of the maximum over the evader's 9 held actions
of the value interpolated (5D multilinear, periodic heading) at the exact
successor after dt -- constant-curvature arcs with speed saturation, as in
pursuit-evasion-core reversible/model.py:86-183.  Two functionals:

* "tube":     V' = min(V, min max V(s')), the capture-by-horizon signed field
              (the same tube convention as the ENO/LF solver); k backups give
              the signed field at horizon k*dt.
* "min_time": u' = 0 in the capture disk, else (1-b) + b min max u(s') with
              b = exp(-dt): value iteration for u = 1 - exp(-T), T the
              minimum capture time.  A contraction, so it converges from any
              start; a good warm start converges in fewer iterations.

The optimal action indices (catalogue order 3*i_a + i_k of
product([-A,0,A],[-K,0,K])) can be recorded with any backup.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .. import _native

MODES = {"tube": _native.PE_SL_TUBE, "min_time": _native.PE_SL_MINTIME}
KERNELS = {"auto": _native.PE_SL_KERNEL_AUTO, "generic": _native.PE_SL_KERNEL_GENERIC,
           "tiled": _native.PE_SL_KERNEL_TILED}


def semilag_params(config, grid, *, dt=0.0, mode="tube", device=0):
    if mode not in MODES:
        raise ValueError("mode must be 'tube' or 'min_time'")
    p, e = config.pursuer, config.evader
    return _native.SemiLagParams(
        positions=grid.positions, headings=grid.headings, p_speeds=grid.p_speeds,
        e_speeds=grid.e_speeds, extent=float(grid.extent),
        capture_radius=float(config.capture_radius),
        p_speed_min=float(p.speed_min), p_speed_max=float(p.speed_max),
        p_acceleration=float(p.acceleration), p_curvature=float(p.max_curvature),
        e_speed_min=float(e.speed_min), e_speed_max=float(e.speed_max),
        e_acceleration=float(e.acceleration), e_curvature=float(e.max_curvature),
        dt=float(dt), mode=MODES[mode], device=int(device))


def interpolation_cfl_dt(config, grid):
    """Largest step that moves no coordinate by more than one spacing."""
    lib = _native.library()
    params = semilag_params(config, grid)
    out = ctypes.c_double()
    _native.check(lib.pe_semilag_dt(ctypes.byref(params), ctypes.byref(out)))
    return out.value


class SemiLagrangianSolver:
    def __init__(self, config, grid, *, dt=0.0, mode="tube", device=0):
        self._lib = _native.library()
        self.grid = grid
        self.mode = mode
        self.shape = tuple(grid.shape)
        self.cells = int(np.prod(self.shape))
        self._params = semilag_params(config, grid, dt=dt, mode=mode, device=device)
        handle = ctypes.c_void_p()
        _native.check(self._lib.pe_semilag_create(ctypes.byref(self._params),
                                                  ctypes.byref(handle)))
        self._h = handle
        out = ctypes.c_double()
        _native.check(self._lib.pe_semilag_dt(ctypes.byref(self._params),
                                              ctypes.byref(out)))
        self.dt = out.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pe_semilag_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def initialize(self, initial=None):
        ptr = None
        if initial is not None:
            initial = np.ascontiguousarray(initial, dtype=np.float32).reshape(-1)
            if initial.size != self.cells:
                raise ValueError("initial field has the wrong number of cells")
            ptr = initial.ctypes.data
        _native.check(self._lib.pe_semilag_init(self._h, ptr))

    def initialize_device(self, device_ptr):
        """Initialise from a dense float32 field already on this device."""
        _native.check(self._lib.pe_semilag_init_device(self._h, ctypes.c_void_p(device_ptr)))

    def track_arrival(self, arrival=None, start_time=0.0):
        """Keep first-crossing times of the tube field from now on: a new
        record (start_time where the value is <= 0) or `arrival` continued."""
        ptr = None
        if arrival is not None:
            arrival = np.ascontiguousarray(arrival, dtype=np.float32).reshape(-1)
            if arrival.size != self.cells:
                raise ValueError("arrival has the wrong number of cells")
            ptr = arrival.ctypes.data
        _native.check(self._lib.pe_semilag_track_arrival(self._h, ptr, float(start_time)))

    def arrival(self, out=None):
        if out is None:
            out = np.empty(self.cells, np.float32)
        _native.check(self._lib.pe_semilag_copy_arrival(self._h, out.ctypes.data))
        return out.reshape(self.shape)

    def backup(self, with_policy=False):
        _native.check(self._lib.pe_semilag_backup(self._h, int(with_policy)))

    def iterate(self, max_iterations, tol=0.0, check_every=1):
        """Value iteration; returns (iterations, last residual, converged)."""
        n, r, c = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int32()
        _native.check(self._lib.pe_semilag_iterate(
            self._h, int(max_iterations), float(tol), int(check_every),
            ctypes.byref(n), ctypes.byref(r), ctypes.byref(c)))
        return n.value, r.value, bool(c.value)

    def residual(self):
        r = ctypes.c_double()
        _native.check(self._lib.pe_semilag_residual(self._h, ctypes.byref(r)))
        return r.value

    def evaluations(self):
        """Action-pair evaluations of the tiled value backups since the last
        initialisation (0 for the generic kernel)."""
        n = ctypes.c_int64()
        _native.check(self._lib.pe_semilag_evaluations(self._h, ctypes.byref(n)))
        return n.value

    def set_skip(self, enable=True):
        """Copy, instead of recomputing, the tiled work items whose
        neighbourhood did not change in the previous backup (exact)."""
        _native.check(self._lib.pe_semilag_set_skip(self._h, int(bool(enable))))

    def items_computed(self):
        """Tiled work items computed (not skipped) since initialisation."""
        n = ctypes.c_int64()
        _native.check(self._lib.pe_semilag_items_computed(self._h, ctypes.byref(n)))
        return n.value

    def value(self, out=None):
        out = np.empty(self.cells, np.float32) if out is None else out
        _native.check(self._lib.pe_semilag_copy_value(self._h, out.ctypes.data))
        return out.reshape(self.shape)

    def value_to_device(self, device_ptr):
        """Copy the value field into a dense float32 array on this device."""
        _native.check(self._lib.pe_semilag_copy_value_device(self._h,
                                                             ctypes.c_void_p(device_ptr)))

    def policy(self):
        p = np.empty(self.cells, np.uint8)
        e = np.empty(self.cells, np.uint8)
        _native.check(self._lib.pe_semilag_copy_policy(self._h, p.ctypes.data,
                                                       e.ctypes.data))
        return p.reshape(self.shape), e.reshape(self.shape)

    def device_value_ptr(self):
        ptr = ctypes.c_void_p()
        _native.check(self._lib.pe_semilag_device_value(self._h, ctypes.byref(ptr)))
        return ptr.value

    def set_stream(self, stream_ptr):
        _native.check(self._lib.pe_semilag_set_stream(self._h, stream_ptr))

    def set_kernel(self, kernel):
        """Value-only backup kernel: "auto" (default), "generic" or "tiled"."""
        if kernel not in KERNELS:
            raise ValueError("kernel must be 'auto', 'generic' or 'tiled'")
        _native.check(self._lib.pe_semilag_set_kernel(self._h, KERNELS[kernel]))

    def set_tile(self, rows):
        """About `rows` cell rows per tiled-kernel work item (0: default)."""
        _native.check(self._lib.pe_semilag_set_tile(self._h, int(rows)))

    @property
    def tile(self):
        r, t, n = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        _native.check(self._lib.pe_semilag_get_tile(self._h, ctypes.byref(r), ctypes.byref(t),
                                                    ctypes.byref(n)))
        return dict(rows=r.value, threads=t.value, items=n.value)

    @property
    def kernel(self):
        k = ctypes.c_int32()
        _native.check(self._lib.pe_semilag_kernel(self._h, ctypes.byref(k)))
        return "tiled" if k.value == _native.PE_SL_KERNEL_TILED else "generic"

    def profile(self, enable=True):
        _native.check(self._lib.pe_semilag_profile(self._h, int(enable)))

    def kernel_time(self):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.pe_semilag_kernel_time(self._h, ctypes.byref(ms),
                                                       ctypes.byref(n)))
        return ms.value, n.value


def capture_time(u):
    """Minimum capture time from the min-time value u = 1 - exp(-T)."""
    u = np.asarray(u, dtype=np.float64)
    with np.errstate(divide="ignore"):
        return np.where(u < 1, -np.log1p(-np.minimum(u, 1)), np.inf)
