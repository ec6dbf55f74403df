"""Compact eight-state semi-Lagrangian contact game, device resident.

Mirrors src/pursuit_evasion/local_game/grid_game.py: the vehicle grid
record (`VehicleGrid`, :21-155), the pair domain (`PairDomain`, :336-381)
and the GPU entry points `gpu_arrays` / `initialize_gpu` / `backup_gpu`
(:226-333) and `packed_gpu_arrays` / `initialize_packed` / `backup_packed`
(:424-581), plus the packed query of local_game/reference.py:122-134
(`query_field`).  Names, arguments, layouts and errors are the reference's;
the work runs in the hand-written kernels of csrc/capi_compact.cu through
the `pe_compact_*` C ABI: one launch per backup with the field resident on
the device (the reference launches two kernels per 256-state chunk and
pursuer action, and in the memory-saving packed mode copies every output
tile through the host).

Grid construction from an arena (`make_grid`, :158-196) asks the vehicle
geometry (legality with a braking backup, held-control arcs, clear
configuration paths) of local_game/engine.py, whose queries run on the GPU
(csrc/vehicle_geometry_exact.cu); a grid bound to that geometry
(`bind_geometry`) falls back, for states without multilinear support, to
their nearest connected grid states (:38-79).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from itertools import product

import numpy as np

from .. import _native

BITS = np.asarray(list(product([0, 1], repeat=4)), np.int64)
STENCIL = 16


@dataclass
class VehicleGrid:
    """One car's legal states [n, 4] (x, y, heading, speed), the dense-to-
    compact map, the controls [na, 2] and the held-control successors:
    16-vertex stencils `successors` / `weights` [n, na, 16], `allowed`
    [n, na] and the retained interpolation mass."""
    axes: tuple
    states: np.ndarray
    dense_to_compact: np.ndarray
    controls: np.ndarray
    successors: np.ndarray
    weights: np.ndarray
    allowed: np.ndarray
    retained_mass: np.ndarray

    def stencil(self, states):
        """Multilinear 16-vertex stencils of 4D states over the legal grid
        (grid_game.py:86-129): periodic heading, clipped positions and
        speeds; weights on omitted vertices are dropped and the rest
        renormalized.  Returns (ids int32, weights float32, valid, shape,
        retained mass).  States without support stay invalid (the
        reference's nearest-supported fallback needs its geometry engine)."""
        s = np.asarray(states, float)
        shape = s.shape[:-1]
        flat = s.reshape(-1, 4)
        inds = np.zeros((len(flat), STENCIL), np.int64)
        w = np.ones((len(flat), STENCIL))
        valid = np.isfinite(flat).all(1)
        sizes = tuple(len(a) for a in self.axes)
        strides = np.cumprod((1,) + sizes[:0:-1])[::-1]
        for k, (axis, stride) in enumerate(zip(self.axes, strides)):
            x = flat[:, k]
            if k == 2:
                f = ((x + np.pi) % (2 * np.pi)) / (2 * np.pi / len(axis))
                j = np.floor(f).astype(np.int64) % len(axis)
                frac = f - np.floor(f)
            else:
                valid &= (x >= axis[0] - 1e-9) & (x <= axis[-1] + 1e-9)
                z = np.clip(x, axis[0], axis[-1])
                j = np.clip(np.searchsorted(axis, z, side="right") - 1, 0, len(axis) - 2)
                frac = (z - axis[j]) / (axis[j + 1] - axis[j])
            coord = j[:, None] + BITS[None, :, k]
            if k == 2:
                coord %= len(axis)
            inds += coord * stride
            w *= np.where(BITS[None, :, k], frac[:, None], 1 - frac[:, None])
        ids = self.dense_to_compact[inds]
        w = np.where(ids >= 0, w, 0)
        mass = w.sum(1)
        missing = valid & (mass <= 1e-9)
        valid &= mass > 1e-9
        w = np.divide(w, mass[:, None], out=np.zeros_like(w), where=mass[:, None] > 1e-9)
        ids = np.maximum(ids, 0).astype(np.int32)
        w = w.astype(np.float32)
        if missing.any() and getattr(self, "_engine", None) is not None:
            unique, inverse = np.unique(flat[missing], axis=0, return_inverse=True)
            inverse = np.asarray(inverse).reshape(-1)
            ni, nw, nv = self._nearest_supported(unique)
            ids[missing], w[missing], valid[missing] = ni[inverse], nw[inverse], nv[inverse]
        return ids, w, valid, shape, mass

    def bind_geometry(self, arena, limits, role, dt=0.05, device=0):
        """Attach the car's geometry: stencils of unsupported states then fall
        back to nearby grid states reachable along a clear straight path."""
        from .engine import GeometryEngine

        self._engine = GeometryEngine(arena, limits, role, control_dt=dt, device=device)
        self._tree = None
        return self

    def _nearest_supported(self, states, neighbours=64):
        """Up to 16 of the `neighbours` nearest grid states (in position,
        heading direction and speed, each scaled by its grid step) that a
        clear straight configuration path reaches, weighted by inverse
        squared feature distance; (ids, weights, valid)."""
        from scipy.spatial import cKDTree

        step_x = self.axes[0][1] - self.axes[0][0]
        step_h = 2 * np.sin(np.pi / len(self.axes[2]))  # chord between headings
        step_v = np.min(np.diff(self.axes[3]))

        def features(s):
            return np.column_stack([s[:, 0] / step_x, s[:, 1] / step_x,
                                    np.cos(s[:, 2]) / step_h, np.sin(s[:, 2]) / step_h,
                                    s[:, 3] / step_v])

        if self._tree is None:
            self._tree = cKDTree(features(self.states))
        k = min(neighbours, len(self.states))
        dist, index = self._tree.query(features(states), k=k)
        dist, index = dist.reshape(len(states), k), index.reshape(len(states), k)
        reach = self._engine.connections(np.repeat(states, k, axis=0),
                                         self.states[index].reshape(-1, 4)).reshape(index.shape)
        # the first 16 reachable neighbours in distance order
        order = np.argsort(~reach, axis=1, kind="stable")[:, :STENCIL]
        keep = np.take_along_axis(reach, order, 1)
        ids = np.where(keep, np.take_along_axis(index, order, 1), 0).astype(np.int32)
        inv = np.where(keep, 1.0 / np.maximum(np.take_along_axis(dist, order, 1), 1e-8) ** 2,
                       0.0)
        total = inv.sum(1, keepdims=True)
        w = np.divide(inv, total, out=np.zeros_like(inv), where=total > 0).astype(np.float32)
        return ids, w, keep.any(1)

    def save(self, path):
        np.savez_compressed(
            path, states=self.states, dense_to_compact=self.dense_to_compact,
            controls=self.controls, successors=self.successors, weights=self.weights,
            allowed=self.allowed, retained_mass=self.retained_mass,
            **{"axis" + str(i): a for i, a in enumerate(self.axes)})

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(tuple(z["axis" + str(i)] for i in range(4)),
                   *[z[k] for k in ("states", "dense_to_compact", "controls", "successors",
                                    "weights", "allowed", "retained_mass")])


def make_grid(arena, limits, role, *, position_step=0.3, headings=8, speeds=None, dt=0.05,
              device=0):
    """One car's vehicle grid in `arena` (grid_game.py:158-196): positions
    every `position_step` across the arena (plus one node beyond each wall),
    `headings` periodic headings from -pi and the given signed speeds; the
    states that are clear with a braking backup are kept, and for each of
    the 9 held controls (acceleration in {-A, 0, A} x curvature in {-K, 0,
    K}) the successor after `dt` with its 16-vertex stencil, allowed where
    the arc is clear, ends backup safe and has support."""
    from .engine import GeometryEngine

    if speeds is None:
        speeds = [-1, 0, 0.5, 1, 2] if role == "pursuer" else [-0.5, 0, 0.25, 0.5, 1]
    cells = int(round(2 * arena.half_width / position_step))
    x = (np.arange(cells + 2) - (cells + 1) / 2) * position_step
    heading = np.arange(headings) * 2 * np.pi / headings - np.pi
    axes = (x, x, heading, np.array(speeds, float))
    lattice = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 4)
    engine = GeometryEngine(arena, limits, role, control_dt=dt, device=device)
    legal = engine.backup_safe(lattice)
    dense_to_compact = np.full(len(lattice), -1, np.int32)
    dense_to_compact[legal] = np.arange(int(legal.sum()), dtype=np.int32)
    kept = lattice[legal]
    A, K = limits.acceleration, limits.max_curvature
    controls = np.array([[a, k] for a in (-A, 0.0, A) for k in (-K, 0.0, K)], float)
    grid = VehicleGrid(axes, kept, dense_to_compact, controls, None, None, None,
                       None).bind_geometry(arena, limits, role, dt, device)
    allowed, successor_states = engine.actions(kept, controls, dt)
    ids, w, supported, _, mass = grid.stencil(successor_states)
    grid.successors = ids.reshape(len(kept), len(controls), STENCIL)
    grid.weights = w.reshape(len(kept), len(controls), STENCIL)
    grid.allowed = allowed & supported.reshape(allowed.shape)
    grid.retained_mass = mass.reshape(allowed.shape)
    if not grid.allowed.any(axis=1).all():
        raise ValueError("A retained state has no legal interpolable action")
    return grid


@dataclass
class PairDomain:
    """Pairs whose centres are within `exit_radius` (grid_game.py:336-381):
    `p_position` [n_p] position class of each pursuer state, `lookup`
    [positions, n_e] rank of an evader state in its class (-1 outside),
    `e_indices` [positions, max_count], `counts` [positions], `offsets`
    [n_p + 1] first pair of each pursuer state in the packed vector."""
    p_position: np.ndarray
    lookup: np.ndarray
    e_indices: np.ndarray
    counts: np.ndarray
    offsets: np.ndarray
    exit_radius: float

    @property
    def states(self):
        return int(self.offsets[-1])

    @classmethod
    def build(cls, p, e, exit_radius=3.0):
        positions, which = np.unique(p.states[:, :2], axis=0, return_inverse=True)
        which = np.asarray(which).reshape(-1)
        lookup = np.full((len(positions), len(e.states)), -1, np.int32)
        members = []
        for i, xy in enumerate(positions):
            ids = np.flatnonzero(np.linalg.norm(e.states[:, :2] - xy, axis=1)
                                 <= exit_radius + 1e-8)
            members.append(ids)
            lookup[i, ids] = np.arange(len(ids), dtype=np.int32)
        counts = np.array([len(x) for x in members], np.int32)
        e_indices = np.zeros((len(positions), int(counts.max())), np.int32)
        for i, ids in enumerate(members):
            e_indices[i, : len(ids)] = ids
        offsets = np.concatenate([[0], np.cumsum(counts[which], dtype=np.int64)])
        return cls(which.astype(np.int32), lookup, e_indices, counts, offsets,
                   float(exit_radius))

    def save(self, path):
        np.savez_compressed(path, p_position=self.p_position, lookup=self.lookup,
                            e_indices=self.e_indices, counts=self.counts,
                            offsets=self.offsets, exit_radius=self.exit_radius)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(*[z[k] for k in ("p_position", "lookup", "e_indices", "counts", "offsets")],
                   float(z["exit_radius"]))


class DeviceField:
    """The current field on the device: `__cuda_array_interface__` for
    zero-copy views (torch.as_tensor(x, device="cuda"), CuPy), `get()` /
    `np.asarray` for a host copy."""

    def __init__(self, arrays):
        self._arrays = arrays

    @property
    def shape(self):
        return (self._arrays.cells,)

    @property
    def dtype(self):
        return np.dtype(np.float32)

    @property
    def __cuda_array_interface__(self):
        ptr = ctypes.c_void_p()
        _native.check(self._arrays._lib.pe_compact_field_device(self._arrays._handle,
                                                                ctypes.byref(ptr)))
        self._arrays.synchronize()
        return {"shape": self.shape, "typestr": "<f4", "data": (ptr.value or 0, False),
                "version": 3, "strides": None}

    def get(self, out=None):
        return self._arrays.field(out)

    def __array__(self, dtype=None, copy=None):
        host = self.get()
        return host if dtype is None else host.astype(dtype)

    def __len__(self):
        return self._arrays.cells


class CompactArrays(dict):
    """Device state of one compact game (the dict of the reference's
    `gpu_arrays`): the pe_compact handle, the field as "current", and the
    reference's bookkeeping keys (memory_bytes, chunk, exit_radius, ...)."""

    def __init__(self, p, e, domain, *, max_gb, chunk, device=0):
        super().__init__()
        self._lib = _native.library()
        self._handle = None
        self._p, self._e, self._domain = p, e, domain
        self._device = device
        n_p, n_e = len(p.states), len(e.states)
        cells = domain.states if domain is not None else n_p * n_e
        grids = sum(_grid_bytes(g) for g in (p, e))
        extra = 0 if domain is None else (domain.lookup.nbytes + domain.e_indices.nbytes)
        row = n_e * 4
        need = cells * 8 + grids + extra + (0 if row <= 192 * 1024 else 148 * 4 * row) + 64 * 2**20
        free = _free_device_bytes(device)
        if need > max_gb * 1e9 or need > free * 0.95:
            raise MemoryError(f"{need/1e9:.2f}GB required; {free/1e9:.2f}GB free")
        self.cells = int(cells)
        self.update(memory_bytes=int(need), chunk=int(chunk))
        self["current"] = DeviceField(self)

    def _create(self, exit_radius):
        if self._handle is not None:
            _native.check(self._lib.pe_compact_destroy(self._handle))
            self._handle = None
        keep = []
        pg, eg = _grid_struct(self._p, keep), _grid_struct(self._e, keep)
        dom = None if self._domain is None else ctypes.byref(_domain_struct(self._domain, keep))
        handle = ctypes.c_void_p()
        _native.check(self._lib.pe_compact_create(ctypes.byref(pg), ctypes.byref(eg), dom,
                                                  float(exit_radius), self._device,
                                                  ctypes.byref(handle)))
        self._handle = handle
        self["exit_radius"] = float(exit_radius)

    def _require(self):
        if self._handle is None:
            raise RuntimeError("initialize the field first")

    def field(self, out=None):
        self._require()
        host = np.empty(self.cells, np.float32) if out is None else out
        if host.dtype != np.float32 or not host.flags.c_contiguous or host.size != self.cells:
            raise ValueError("out must be a contiguous float32 array of the field's size")
        _native.check(self._lib.pe_compact_copy_field(self._handle, host.ctypes.data,
                                                      self.cells))
        return host

    def set_field(self, values):
        self._require()
        host = np.ascontiguousarray(values, np.float32).reshape(-1)
        _native.check(self._lib.pe_compact_set_field(self._handle, host.ctypes.data,
                                                     host.size))

    def backup(self, count=1):
        self._require()
        _native.check(self._lib.pe_compact_backup(self._handle, int(count)))

    def synchronize(self):
        if self._handle is not None:
            _native.check(self._lib.pe_compact_synchronize(self._handle))

    def set_stream(self, stream_ptr):
        self._require()
        _native.check(self._lib.pe_compact_set_stream(self._handle, stream_ptr))

    def profile(self, enable=True):
        self._require()
        _native.check(self._lib.pe_compact_profile(self._handle, int(enable)))

    def kernel_time(self):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.pe_compact_kernel_time(self._handle, ctypes.byref(ms),
                                                       ctypes.byref(n)))
        return ms.value, n.value

    def query(self, pi, pw, ei, ew):
        self._require()
        arrays = [np.ascontiguousarray(pi, np.int32), np.ascontiguousarray(pw, np.float32),
                  np.ascontiguousarray(ei, np.int32), np.ascontiguousarray(ew, np.float32)]
        n = len(arrays[0])
        for a in arrays:
            if a.shape != (n, STENCIL):
                raise ValueError("query stencils must be [n, 16]")
        out = np.empty(n, np.float32)
        _native.check(self._lib.pe_compact_query(self._handle, n, *(a.ctypes.data for a in arrays),
                                                 out.ctypes.data))
        return out

    def close(self):
        if self._handle is not None:
            _native.check(self._lib.pe_compact_destroy(self._handle))
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _grid_bytes(g):
    return g.successors.size * 8 + g.allowed.size + g.states.size * 4


def _free_device_bytes(device):
    try:
        import torch

        if torch.cuda.is_available():
            free, _ = torch.cuda.mem_get_info(device)
            return free
    except Exception:
        pass
    return float("inf")


def _grid_struct(g, keep):
    n, na = g.allowed.shape
    arrays = [np.ascontiguousarray(g.states, np.float32).reshape(n, 4),
              np.ascontiguousarray(g.successors, np.int32).reshape(n, na, STENCIL),
              np.ascontiguousarray(g.weights, np.float32).reshape(n, na, STENCIL),
              np.ascontiguousarray(g.allowed, np.uint8).reshape(n, na)]
    keep.extend(arrays)
    return _native.VehicleGridArrays(n, na, *(a.ctypes.data for a in arrays))


def _domain_struct(d, keep):
    arrays = [np.ascontiguousarray(d.p_position, np.int32),
              np.ascontiguousarray(d.lookup, np.int32),
              np.ascontiguousarray(d.e_indices, np.int32),
              np.ascontiguousarray(d.counts, np.int32),
              np.ascontiguousarray(d.offsets, np.int64)]
    keep.extend(arrays)
    return _native.PairDomainArrays(len(d.counts), d.e_indices.shape[1],
                                    *(a.ctypes.data for a in arrays))


# ---------------------------------------------------------------- dense layout
def gpu_arrays(p, e, *, max_gb=7.6, chunk=256, device=0):
    """Device state for the dense [n_p * n_e] field (grid_game.py:226-251).
    MemoryError when the working set exceeds `max_gb` or 95 % of the free
    device memory.  `chunk` is kept for the reference's signature: a backup
    is one launch over every pursuer state."""
    return CompactArrays(p, e, None, max_gb=max_gb, chunk=chunk, device=device)


def initialize_gpu(a, p, e, arena, exit_radius=3.0):
    """Capture field (rectangle contact of the arena's footprints), the exit
    radius where the centres are farther apart (grid_game.py:254-283)."""
    a._create(exit_radius)
    _native.check(a._lib.pe_compact_init(a._handle, arena.pursuer.length,
                                         arena.pursuer.width, arena.evader.length,
                                         arena.evader.width))


def backup_gpu(a, p, e):
    """One min-max backup of the dense field (grid_game.py:286-333)."""
    a.backup(1)


# --------------------------------------------------------------- packed layout
def packed_gpu_arrays(p, e, domain, *, max_gb=7.6, chunk=256, tiled_output=False, device=0):
    """Device state for the pair-packed field (grid_game.py:424-481).  The
    field stays on the device; `tiled_output` (the reference's host-staged
    output tiles) is accepted for its signature and needs no host buffer."""
    a = CompactArrays(p, e, domain, max_gb=max_gb, chunk=chunk, device=device)
    a._create(domain.exit_radius)
    a.update(tiled_output=bool(tiled_output))
    return a


def initialize_packed(a, p, e, domain, arena):
    """Capture field of every pair of the domain (grid_game.py:484-509)."""
    _native.check(a._lib.pe_compact_init(a._handle, arena.pursuer.length,
                                         arena.pursuer.width, arena.evader.length,
                                         arena.evader.width))


def backup_packed(a, p, e, domain):
    """One min-max backup of the packed field (grid_game.py:512-581)."""
    a.backup(1)


def query_field(a, pi, pw, ei, ew):
    """Values at product stencils (pursuer ids/weights [n, 16], evader
    ids/weights [n, 16]) of the current field (reference.py:122-134)."""
    return a.query(pi, pw, ei, ew)
