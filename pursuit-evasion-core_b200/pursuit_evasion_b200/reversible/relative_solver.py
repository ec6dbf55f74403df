"""Owning Python handle of the relative 5D CUDA solver (pe_relative_* C ABI).

One RelativeSolver = one device-resident field, stage buffer and arrival
array on one GPU.  It is what `free_dp.solve` drives frame by frame, and the
object a caller uses to run the hot path without the table-writing driver
(benchmarks, warm starts, convergence runs).
"""

from __future__ import annotations

import ctypes

import numpy as np

from .. import _native


def _params(config, grid, *, order, cfl, precision, device):
    p, e = config.pursuer, config.evader
    return _native.RelativeParams(
        positions=int(grid.positions),
        headings=int(grid.headings),
        p_speeds=int(grid.p_speeds),
        e_speeds=int(grid.e_speeds),
        extent=float(grid.extent),
        capture_radius=float(config.capture_radius),
        p_speed_min=float(p.speed_min),
        p_speed_max=float(p.speed_max),
        p_acceleration=float(p.acceleration),
        p_curvature=float(p.max_curvature),
        e_speed_min=float(e.speed_min),
        e_speed_max=float(e.speed_max),
        e_acceleration=float(e.acceleration),
        e_curvature=float(e.max_curvature),
        cfl=float(cfl),
        order=int(order),
        scheme=_native.PE_SCHEME_ENO_LF,
        precision=precision,
        device=int(device),
    )


PRECISIONS = {"float32": _native.PE_LOCAL_F32, "float64": _native.PE_LOCAL_F64}


def cfl_limit(config, grid, *, order=2, cfl=0.8):
    """The reference's CFL step limit (native_relative.cpp:70-81)."""
    lib = _native.library()
    params = _params(config, grid, order=order, cfl=cfl,
                     precision=_native.PE_LOCAL_F32, device=0)
    out = ctypes.c_double()
    _native.check(lib.pe_relative_cfl_limit(ctypes.byref(params), ctypes.byref(out)))
    return out.value


class RelativeSolver:
    def __init__(self, config, grid, *, order=2, cfl=0.8,
                 local_precision="float32", device=0):
        if local_precision not in PRECISIONS:
            raise ValueError("local_precision must be float32 or float64")
        self._lib = _native.library()
        self.grid = grid
        self.shape = tuple(grid.shape)
        self.cells = int(np.prod(self.shape))
        self.local_precision = local_precision
        self._params = _params(config, grid, order=order, cfl=cfl,
                               precision=PRECISIONS[local_precision],
                               device=device)
        handle = ctypes.c_void_p()
        _native.check(self._lib.pe_relative_create(ctypes.byref(self._params),
                                                   ctypes.byref(handle)))
        self._h = handle
        limit = ctypes.c_double()
        _native.check(self._lib.pe_relative_cfl_limit(ctypes.byref(self._params),
                                                      ctypes.byref(limit)))
        self.cfl_dt_limit = limit.value

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.pe_relative_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state ------------------------------------------------------------
    def initialize(self, initial=None, arrival=None, start_time=0.0):
        """Circular capture field when `initial` is None, else a full field."""
        ptr_i = ptr_a = None
        keep = []
        if initial is not None:
            initial = np.ascontiguousarray(initial, dtype=np.float32).reshape(-1)
            if initial.size != self.cells:
                raise ValueError("initial field has the wrong number of cells")
            keep.append(initial)
            ptr_i = initial.ctypes.data
        if arrival is not None:
            arrival = np.ascontiguousarray(arrival, dtype=np.float32).reshape(-1)
            if arrival.size != self.cells:
                raise ValueError("arrival has the wrong number of cells")
            keep.append(arrival)
            ptr_a = arrival.ctypes.data
        _native.check(self._lib.pe_relative_init(self._h, ptr_i, ptr_a,
                                                 float(start_time)))

    def initialize_plane(self, plane, start_time=0.0):
        """Field = `plane` repeated over the outer axes (gpu_relative.py:42-45):
        a (y, x) plane or a (psi, y, x) block in storage order."""
        plane = np.ascontiguousarray(plane, dtype=np.float32).reshape(-1)
        _native.check(self._lib.pe_relative_init_plane(self._h, plane.ctypes.data,
                                                       plane.size, float(start_time)))

    def set_exit(self, radius):
        """Local exit (gpu_relative.py:96-101): cells with x^2 + y^2 > radius^2
        are held at `radius` and never arrive.  The reference bakes radius^2
        and radius into its kernel as 10-significant-digit literals; the same
        rounded numbers are passed here.  None disables the exit."""
        if radius is None:
            r = r2 = 0.0
        else:
            radius = float(radius)
            r, r2 = float(f"{radius:.9e}"), float(f"{radius ** 2:.9e}")
        _native.check(self._lib.pe_relative_set_exit(self._h, r, r2))

    def probe(self, indices, weights):
        """sum_k weights[i, k] * field[indices[i, k]] over 32-corner stencils
        (dense storage-order indices), summed in double on the device."""
        indices = np.ascontiguousarray(indices, dtype=np.int64)
        weights = np.ascontiguousarray(weights, dtype=np.float64)
        if indices.ndim != 2 or indices.shape[1] != 32 or weights.shape != indices.shape:
            raise ValueError("probe stencils must be [n, 32] index and weight arrays")
        out = np.empty(len(indices), np.float64)
        _native.check(self._lib.pe_relative_probe(self._h, len(indices), indices.ctypes.data,
                                                  weights.ctypes.data, out.ctypes.data))
        return out

    def set_stream(self, stream_ptr):
        _native.check(self._lib.pe_relative_set_stream(self._h, stream_ptr))

    def advance(self, goal):
        steps = ctypes.c_int64()
        _native.check(self._lib.pe_relative_advance(self._h, float(goal),
                                                    ctypes.byref(steps)))
        return steps.value

    def step(self, dt):
        _native.check(self._lib.pe_relative_step(self._h, float(dt)))

    @property
    def time(self):
        t = ctypes.c_double()
        n = ctypes.c_int64()
        _native.check(self._lib.pe_relative_time(self._h, ctypes.byref(t),
                                                 ctypes.byref(n)))
        return t.value

    @property
    def steps(self):
        t = ctypes.c_double()
        n = ctypes.c_int64()
        _native.check(self._lib.pe_relative_time(self._h, ctypes.byref(t),
                                                 ctypes.byref(n)))
        return n.value

    def synchronize(self):
        _native.check(self._lib.pe_relative_synchronize(self._h))

    def field(self, out=None):
        if out is None:
            out = np.empty(self.cells, np.float32)
        _native.check(self._lib.pe_relative_copy_field(self._h, out.ctypes.data))
        return out.reshape(self.shape)

    def copy_field_to(self, host_ptr):
        """Device-to-host copy into a caller buffer (e.g. pinned memory)."""
        _native.check(self._lib.pe_relative_copy_field(self._h, host_ptr))

    def arrival(self, out=None):
        if out is None:
            out = np.empty(self.cells, np.float32)
        _native.check(self._lib.pe_relative_copy_arrival(self._h, out.ctypes.data))
        return out.reshape(self.shape)

    def snapshot(self, slot):
        """Enqueue a copy of the current field into snapshot buffer `slot`
        (0 or 1) on the solver's stream; returns at once."""
        _native.check(self._lib.pe_relative_snapshot(self._h, int(slot)))

    def copy_snapshot(self, slot, host_ptr):
        """Copy snapshot `slot` to host memory once it is complete (on a
        separate copy stream; callable from another thread while the solver
        advances)."""
        _native.check(self._lib.pe_relative_copy_snapshot(self._h, int(slot), host_ptr))

    def device_field_ptr(self):
        ptr = ctypes.c_void_p()
        _native.check(self._lib.pe_relative_device_field(self._h, ctypes.byref(ptr)))
        return ptr.value

    @property
    def tile(self):
        """(rows, psi_chunk) of the float32 stage kernel."""
        rows, chunk = ctypes.c_int32(), ctypes.c_int32()
        _native.check(self._lib.pe_relative_get_tile(self._h, ctypes.byref(rows),
                                                     ctypes.byref(chunk)))
        return rows.value, chunk.value

    def set_tile(self, rows, psi_chunk):
        _native.check(self._lib.pe_relative_set_tile(self._h, int(rows),
                                                     int(psi_chunk)))

    def kernel_info(self):
        """(threads per CTA, shared bytes per CTA, resident CTAs per SM)."""
        vals = [ctypes.c_int32() for _ in range(3)]
        _native.check(self._lib.pe_relative_kernel_info(self._h, *map(ctypes.byref, vals)))
        return tuple(v.value for v in vals)

    def stats(self):
        """(residual of the last step, maximum increase since init)."""
        r = ctypes.c_double()
        inc = ctypes.c_double()
        _native.check(self._lib.pe_relative_stats(self._h, ctypes.byref(r),
                                                  ctypes.byref(inc)))
        return r.value, inc.value

    def profile(self, enable=True):
        _native.check(self._lib.pe_relative_profile(self._h, int(enable)))

    def kernel_time(self, stage):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        _native.check(self._lib.pe_relative_kernel_time(self._h, int(stage),
                                                        ctypes.byref(ms),
                                                        ctypes.byref(n)))
        return ms.value, n.value


class PinnedBuffer:
    """Page-locked host float32 buffer (pe_host_alloc) with a NumPy view."""

    def __init__(self, count):
        self._lib = _native.library()
        ptr = ctypes.c_void_p()
        _native.check(self._lib.pe_host_alloc(ctypes.c_size_t(4 * int(count)), ctypes.byref(ptr)))
        self.ptr = ptr.value
        self.array = np.ctypeslib.as_array((ctypes.c_float * int(count)).from_address(self.ptr))

    def close(self):
        if self.ptr:
            self.array = None
            _native.check(self._lib.pe_host_free(ctypes.c_void_p(self.ptr)))
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
