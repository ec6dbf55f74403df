"""FP64-storage relative 5D solve on the GPU, and the error of a float32
table against it.

The reference stores its tables in float32 (native_relative.cpp:82-83); its
CPU restatement with double storage is the FP64 oracle (po_rel_stage_f64 in
oracle/relative5d.c).  `RelativeSolverF64` runs that same exact stage with
double values on the GPU (pe_relative_f64_* C ABI), bit for bit equal to
the oracle, so the error of a float32 table can be measured at sizes the
CPU cannot reach: `subsampled_error` compares two fields on every `step`-th
node of x, y and psi and every speed (the "1/8-subsampled tile" at
step 8).
"""

from __future__ import annotations

import ctypes

import numpy as np

from .. import _native
from .relative_solver import _params


class RelativeSolverF64:
    def __init__(self, config, grid, *, order=2, cfl=0.8, device=0):
        self._lib = _native.library()
        self.grid = grid
        self.shape = tuple(grid.shape)
        self.cells = int(np.prod(self.shape))
        params = _params(config, grid, order=order, cfl=cfl,
                         precision=_native.PE_LOCAL_F64, device=device)
        handle = ctypes.c_void_p()
        _native.check(self._lib.pe_relative_f64_create(ctypes.byref(params),
                                                       ctypes.byref(handle)))
        self._h = handle

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pe_relative_f64_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, cuda_stream):
        _native.check(self._lib.pe_relative_f64_set_stream(self._h, cuda_stream))

    def initialize(self):
        """V0 = hypot(x, y) - capture_radius in double."""
        _native.check(self._lib.pe_relative_f64_initialize(self._h))

    def step(self, dt):
        _native.check(self._lib.pe_relative_f64_step(self._h, float(dt)))

    def advance(self, goal):
        taken = ctypes.c_int64()
        _native.check(self._lib.pe_relative_f64_advance(self._h, float(goal),
                                                        ctypes.byref(taken)))
        return taken.value

    def _time(self):
        t, steps, limit = ctypes.c_double(), ctypes.c_int64(), ctypes.c_double()
        _native.check(self._lib.pe_relative_f64_time(self._h, ctypes.byref(t),
                                                     ctypes.byref(steps),
                                                     ctypes.byref(limit)))
        return t.value, steps.value, limit.value

    @property
    def time(self):
        return self._time()[0]

    @property
    def steps(self):
        return self._time()[1]

    @property
    def cfl_dt_limit(self):
        return self._time()[2]

    def residual(self):
        out = ctypes.c_double()
        _native.check(self._lib.pe_relative_f64_stats(self._h, ctypes.byref(out)))
        return out.value

    def field(self):
        out = np.empty(self.shape, np.float64)
        _native.check(self._lib.pe_relative_f64_copy_field(self._h, out.ctypes.data))
        return out


def subsample(field, step=8):
    """Nodes (vP, vE, psi, y, x) of a table field at every `step`-th x, y
    and psi index (from 0) and every speed."""
    field = np.asarray(field)
    return field[:, :, ::step, ::step, ::step]


def subsampled_error(table, reference, step=8):
    """Error of `table` (float32 storage) against `reference` (FP64) on the
    subsampled nodes: max-abs, 99.9th percentile, mean and the node count."""
    a = subsample(table, step).astype(np.float64)
    b = subsample(reference, step)
    err = np.abs(a - b).ravel()
    return {"max_abs": float(err.max()), "p999_abs": float(np.quantile(err, 0.999)),
            "mean_abs": float(err.mean()), "nodes": int(err.size), "step": int(step)}
