"""A vP-slab shard whose stage is the CPU oracle (test infrastructure only).

It has the interface of pursuit_evasion_b200.reversible.sharded.RelativeShard
(layout, stage, slabs, field, arrival, stats) over host arrays, so the
sharding driver and its halo exchanges (in-process and torch.distributed
with gloo) run on CPU.  A stage evaluates the oracle on the whole grid with
every slab outside this shard's buffer set to a huge sentinel, and keeps the
owned slabs: a missing or stale halo slab changes the owned values, so
agreement with the unsharded oracle shows that the exchanges deliver
exactly the slabs the stencil reads."""

import ctypes

import numpy as np

SENTINEL = np.float32(1e20)


class OracleShard:
    def __init__(self, oracle, config, grid, vp_begin, vp_end, *, order=2, cfl=0.8):
        self.oracle = oracle
        self.cfg = oracle.rel_cfg(config, grid, order=order, cfl=cfl)
        self.grid, self.order, self.device = grid, order, None
        nvp = grid.p_speeds
        lo, hi = max(0, vp_begin - order), min(nvp, vp_end + order)
        self.layout = (lo, hi, vp_begin, vp_end)
        self.slab_cells = self.slab_floats = grid.states // nvp
        n = (hi - lo) * self.slab_cells
        self.a = np.zeros(n, np.float32)
        self.b = np.zeros(n, np.float32)
        self._arr = np.full(n, np.nan, np.float32)
        self.last = self.a
        self.t = 0.0
        self.residual = self.increase = 0.0
        self.cfl_dt_limit = oracle.rel_cfl_limit(self.cfg)

    def _own(self):
        lo, _, own_lo, own_hi = self.layout
        S = self.slab_cells
        return slice((own_lo - lo) * S, (own_hi - lo) * S), slice(own_lo * S, own_hi * S)

    def initialize(self, initial=None, start_time=0.0):
        lo, hi = self.layout[:2]
        S = self.slab_cells
        if initial is None:
            field = np.zeros(self.grid.states, np.float32)
            arrival = np.zeros(self.grid.states, np.float32)
            self.oracle.lib.po_rel_init(ctypes.addressof(self.cfg), field.ctypes.data,
                                        arrival.ctypes.data)
            initial = field
        initial = np.asarray(initial, np.float32).reshape(-1)[lo * S:hi * S]
        self.a[:] = initial
        self._arr[:] = np.where(initial <= 0, np.float32(start_time), np.float32(np.nan))
        self.last, self.t = self.a, float(start_time)

    def stage(self, k, dt):
        lo, hi = self.layout[:2]
        S, N = self.slab_cells, self.grid.states
        blend = k == 1
        src, dst = (self.b, self.a) if blend else (self.a, self.b)
        full_src = np.full(N, SENTINEL, np.float32)
        full_dst = np.full(N, SENTINEL, np.float32)
        full_arr = np.full(N, np.nan, np.float32)
        full_src[lo * S:hi * S] = src
        full_dst[lo * S:hi * S] = dst
        full_arr[lo * S:hi * S] = self._arr
        own, gown = self._own()
        prev = (dst if blend else src)[own].astype(np.float64)
        rc, _ = self.oracle.rel_stage_f32(self.cfg, full_src, full_dst, full_arr, dt, self.t,
                                          int(blend))
        assert rc == 0, rc
        dst[own] = full_dst[gown]
        self._arr[own] = full_arr[gown]
        self.last = dst
        if k == self.order - 1:
            change = dst[own].astype(np.float64) - prev
            self.residual = float(np.abs(change).max(initial=0.0))
            self.increase = float(np.maximum(change, 0).max(initial=0.0))
            if self.order == 1:
                self.a, self.b = self.b, self.a
            self.t += dt

    def slabs(self, first, last):
        import torch

        lo = self.layout[0]
        S = self.slab_cells
        return torch.from_numpy(self.last[(first - lo) * S:(last - lo) * S])

    def field(self):
        return self.a[self._own()[0]].copy()

    def arrival(self):
        return self._arr[self._own()[0]].copy()

    def stats(self):
        return self.residual, self.increase
