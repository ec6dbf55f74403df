"""vP-slab sharding of the relative 5D ENO/LF solve (pe_relative_shard_*).

The table's storage order [vP, vE, psi, y, x] makes each pursuer-speed
index one contiguous slab, so a grid too large for one GPU splits into
contiguous slab ranges, one per GPU.  The ENO stencil along vP reaches
`order` slabs, so every shard keeps `order` halo slabs on each side that has
a neighbour, and after every stage the edge slabs of the buffer just written
travel to the neighbours: `LocalExchange` for shards in one process (device
copies), `DistExchange` for one shard per rank (torch.distributed P2P; NCCL
over NVLink on GPUs).  The residual is the maximum over shards.  Each cell
is updated by the single-grid stage of the chosen precision, so a sharded
solve equals the single-grid solve bit for bit (with float64 local
arithmetic, also the reference executable).

The reference solves one grid in one process (native_relative.cpp:173-190);
it has no sharded solve.
"""

from __future__ import annotations

import ctypes
import json
from pathlib import Path

import numpy as np

from .. import _native
from .relative_solver import PRECISIONS, _params, cfl_limit


def partition(p_speeds, parts, order=2):
    """Contiguous owned vP ranges [(begin, end)] of near-equal size; every
    part owns at least `order` slabs when there is more than one."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    if parts > 1 and p_speeds < parts * order:
        raise ValueError(f"{p_speeds} vP slabs cannot give {parts} shards of >= {order} slabs")
    base, extra = divmod(p_speeds, parts)
    out, begin = [], 0
    for k in range(parts):
        end = begin + base + (1 if k < extra else 0)
        out.append((begin, end))
        begin = end
    return out


def halo_plan(layout, order, p_speeds):
    """Slab ranges (global indices) to send and receive on each side:
    {"lower": (send, recv), "upper": (send, recv)} for the sides that have a
    neighbour.  A lower neighbour's upper halo is this shard's first
    `order` owned slabs, and the reverse."""
    lo, hi, own_lo, own_hi = layout
    plan = {}
    if own_lo > 0:
        plan["lower"] = ((own_lo, own_lo + order), (lo, own_lo))
    if own_hi < p_speeds:
        plan["upper"] = ((own_hi - order, own_hi), (own_hi, hi))
    return plan


class _DeviceSlabs:
    """`__cuda_array_interface__` over consecutive slabs of a shard buffer."""

    def __init__(self, ptr, count):
        self._ptr, self._count = ptr, count

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self._count,), "typestr": "<f4", "data": (self._ptr, False),
                "version": 3, "strides": None}


class RelativeShard:
    """One shard on one GPU: owned global vP slabs [vp_begin, vp_end)."""

    def __init__(self, config, grid, vp_begin, vp_end, *, order=2, cfl=0.8,
                 local_precision="float64", device=0):
        if local_precision not in PRECISIONS:
            raise ValueError("local_precision must be float32 or float64")
        self._lib = _native.library()
        self.grid = grid
        self.order = order
        self.device = device
        self._params = _params(config, grid, order=order, cfl=cfl,
                               precision=PRECISIONS[local_precision], device=device)
        handle = ctypes.c_void_p()
        _native.check(self._lib.pe_relative_shard_create(
            ctypes.byref(self._params), int(vp_begin), int(vp_end), ctypes.byref(handle)))
        self._h = handle
        slabs = (ctypes.c_int32 * 4)()
        floats = ctypes.c_int64()
        _native.check(self._lib.pe_relative_shard_layout(self._h, slabs, ctypes.byref(floats)))
        self.layout = tuple(int(v) for v in slabs)
        self.slab_floats = floats.value
        self.slab_cells = grid.e_speeds * grid.headings * grid.positions ** 2
        self.cfl_dt_limit = cfl_limit(config, grid, order=order, cfl=cfl)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pe_relative_shard_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_ptr):
        _native.check(self._lib.pe_relative_shard_set_stream(self._h, stream_ptr))

    def initialize(self, initial=None, start_time=0.0):
        """The circular capture field, or `initial`: the whole dense grid
        (its buffer slabs are taken) or just buffer slabs [lo, hi)."""
        ptr, keep = None, None
        if initial is not None:
            lo, hi = self.layout[:2]
            initial = np.asarray(initial, dtype=np.float32).reshape(-1)
            if initial.size == self.grid.states:
                initial = initial[lo * self.slab_cells:hi * self.slab_cells]
            if initial.size != (hi - lo) * self.slab_cells:
                raise ValueError("initial must hold the grid or the shard's buffer slabs")
            keep = np.ascontiguousarray(initial)
            ptr = keep.ctypes.data
        _native.check(self._lib.pe_relative_shard_init(self._h, ptr, float(start_time)))

    def stage(self, k, dt):
        _native.check(self._lib.pe_relative_shard_stage(self._h, int(k), float(dt)))

    def slabs(self, first, last):
        """Zero-copy device view (torch) of global slabs [first, last) of the
        buffer the last stage wrote."""
        import torch

        ptr = ctypes.c_void_p()
        _native.check(self._lib.pe_relative_shard_buffer(self._h, ctypes.byref(ptr)))
        offset = (first - self.layout[0]) * self.slab_floats * 4
        view = _DeviceSlabs(ptr.value + offset, (last - first) * self.slab_floats)
        return torch.as_tensor(view, device=f"cuda:{self.device}")

    def field(self):
        lo, hi, own_lo, own_hi = self.layout
        out = np.empty((own_hi - own_lo) * self.slab_cells, np.float32)
        _native.check(self._lib.pe_relative_shard_copy_field(self._h, out.ctypes.data))
        return out

    def arrival(self):
        lo, hi, own_lo, own_hi = self.layout
        out = np.empty((own_hi - own_lo) * self.slab_cells, np.float32)
        _native.check(self._lib.pe_relative_shard_copy_arrival(self._h, out.ctypes.data))
        return out

    def stats(self):
        r, inc = ctypes.c_double(), ctypes.c_double()
        _native.check(self._lib.pe_relative_shard_stats(self._h, ctypes.byref(r),
                                                        ctypes.byref(inc)))
        return r.value, inc.value

    def synchronize(self):
        _native.check(self._lib.pe_relative_shard_synchronize(self._h))


class LocalExchange:
    """Halo refresh between shards held by this process (device copies on
    the current stream)."""

    def __init__(self, shards):
        self.shards = list(shards)

    def __call__(self):
        for left, right in zip(self.shards[:-1], self.shards[1:]):
            p_speeds = left.grid.p_speeds
            (l_send, l_recv) = halo_plan(left.layout, left.order, p_speeds)["upper"]
            (r_send, r_recv) = halo_plan(right.layout, right.order, p_speeds)["lower"]
            right.slabs(*r_recv).copy_(left.slabs(*l_send))
            left.slabs(*l_recv).copy_(right.slabs(*r_send))

    def max_residual(self):
        return max(s.stats()[0] for s in self.shards)


class DistExchange:
    """Halo refresh with the neighbouring ranks (one shard per rank, rank r
    holding the r-th range of `partition`) by torch.distributed P2P."""

    def __init__(self, shard, group=None):
        import torch.distributed as dist

        self.dist, self.group = dist, group
        self.shard = shard
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def __call__(self):
        dist = self.dist
        plan = halo_plan(self.shard.layout, self.shard.order, self.shard.grid.p_speeds)
        ops, recvs = [], []
        for side, peer in (("lower", self.rank - 1), ("upper", self.rank + 1)):
            if side not in plan:
                continue
            send, recv = plan[side]
            global_peer = dist.get_global_rank(self.group, peer) if self.group else peer
            buf = self.shard.slabs(*recv)
            ops.append(dist.P2POp(dist.isend, self.shard.slabs(*send).contiguous(),
                                  global_peer, self.group))
            ops.append(dist.P2POp(dist.irecv, buf, global_peer, self.group))
            recvs.append(buf)
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def max_residual(self):
        import torch

        r = torch.tensor([self.shard.stats()[0]], dtype=torch.float64,
                         device=_stat_device(self.shard))
        self.dist.all_reduce(r, op=self.dist.ReduceOp.MAX, group=self.group)
        return float(r.item())


def _stat_device(shard):
    return f"cuda:{shard.device}" if isinstance(shard, RelativeShard) else "cpu"


class ShardedSolver:
    """Steps a set of shards (all of this process's shards, or this rank's
    one) in lock step: each stage on every shard, then the halo exchange.
    GPU shards (all on one device) share one torch stream with the
    exchanges, so stages and copies or NCCL transfers are ordered without
    host synchronisation."""

    def __init__(self, shards, exchange, *, start_time=0.0):
        self.shards = list(shards)
        self.exchange = exchange
        self.time = float(start_time)
        self.steps = 0
        self.order = self.shards[0].order
        self.cfl_dt_limit = self.shards[0].cfl_dt_limit
        self._stream = None
        gpu = [s for s in self.shards if isinstance(s, RelativeShard)]
        if gpu:
            import torch

            if len({s.device for s in gpu}) != 1:
                raise ValueError("the shards of one process must share one device")
            self._stream = torch.cuda.Stream(device=gpu[0].device)
            for s in gpu:
                s.set_stream(self._stream.cuda_stream)

    def step(self, dt):
        if self._stream is None:
            self._step(dt)
        else:
            import torch

            with torch.cuda.stream(self._stream):
                self._step(dt)

    def _step(self, dt):
        for k in range(self.order):
            for s in self.shards:
                s.stage(k, dt)
            self.exchange()
        self.time += dt
        self.steps += 1

    def advance(self, goal):
        """Steps of the CFL limit (the last one shorter) up to `goal`, as
        native_relative.cpp:173-190 takes them."""
        while self.time < goal - 1e-12:
            self.step(min(self.cfl_dt_limit, goal - self.time))

    def residual(self):
        if self._stream is None:
            return self.exchange.max_residual()
        import torch

        with torch.cuda.stream(self._stream):
            return self.exchange.max_residual()


def _agree(error, group, what):
    """Every rank of `group` learns whether any rank failed at this point.
    The failing rank re-raises its own exception; the others raise
    RuntimeError naming the first failing rank.  Each rank takes this
    collective at the same points, so it never waits on a rank that left."""
    import torch.distributed as dist

    reports = [None] * dist.get_world_size(group)
    dist.all_gather_object(reports, None if error is None else repr(error), group=group)
    if error is not None:
        raise error
    failed = [(r, msg) for r, msg in enumerate(reports) if msg is not None]
    if failed:
        r, msg = failed[0]
        raise RuntimeError(f"rank {r} failed during {what}: {msg}")


def solve(config, grid, output, *, horizon=2.0, output_dt=0.1, order=2, cfl=0.8,
          local_precision="float64", history=True, device=None, group=None,
          shard_factory=None):
    """The table directory of free_dp.solve (same files and layout, read by
    RelativeTable) computed by one vP shard per rank of an initialised
    torch.distributed group.  Every rank writes its own slabs of each frame
    into the shared files (the ranks share a file system, as the GPUs of one
    node do); rank 0 creates the directory and writes meta.json.
    `shard_factory(begin, end)` replaces the GPU shard (tests use it)."""
    import os
    import time

    import torch.distributed as dist

    from .free_dp import SCHEMA, _validate, output_times, physics_signature
    from .model import config_dict

    started = time.perf_counter()
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    _validate(config, grid, horizon, output_dt, order, cfl, 1)
    ranges = partition(grid.p_speeds, world, order)
    begin, end = ranges[rank]
    output = Path(output).resolve()
    times = output_times(horizon, output_dt)
    N = grid.states
    files = {"final.f32": N * 4, "arrival.f32": N * 4}
    if history:
        files["fields.f32"] = N * 4 * len(times)
    error = None
    if rank == 0:
        try:
            if output.exists() and any(output.iterdir()):
                raise FileExistsError(f"Preserve existing output: {output}")
            output.mkdir(parents=True, exist_ok=True)
            for name, size in files.items():
                with (output / name).open("wb") as f:
                    f.truncate(size)
        except Exception as exc:  # every rank learns of it before any work
            error = exc
    flag = [error is None]
    dist.broadcast_object_list(flag, src=dist.get_global_rank(group, 0) if group else 0,
                               group=group)
    if error is not None:
        raise error
    if not flag[0]:
        raise RuntimeError("rank 0 could not create the output directory")
    if shard_factory is None:
        import torch

        dev = torch.cuda.current_device() if device is None else device

        def shard_factory(b, e):
            return RelativeShard(config, grid, b, e, order=order, cfl=cfl,
                                 local_precision=local_precision, device=dev)

    shard = None
    fds = {}
    try:
        # Set-up (the shard's device buffers, the initial field, the files):
        # a rank that fails here tells the others before any collective of
        # the solve, so no rank waits on a peer that has left.
        error = None
        try:
            shard = shard_factory(begin, end)
            shard.initialize()
            solver = ShardedSolver([shard], DistExchange(shard, group))
            slab_bytes = (N // grid.p_speeds) * 4
            offset = begin * slab_bytes
            fds = {name: os.open(output / name, os.O_WRONLY) for name in files}
        except Exception as exc:
            error = exc
        _agree(error, group, "shard set-up")

        def put(name, values, base=0):
            os.pwrite(fds[name], np.ascontiguousarray(values, np.float32).tobytes(),
                      base + offset)

        # Frames: every rank reports after each frame (one small collective
        # per frame), so a failure in a frame's steps or its write stops every
        # rank at that frame boundary.
        update = 0.0
        for k, goal in enumerate(times, start=0):
            error = None
            try:
                if k > 0:
                    t0 = time.perf_counter()
                    solver.advance(goal)
                    update += time.perf_counter() - t0
                if history:
                    put("fields.f32", shard.field(), k * N * 4)
                if k == len(times) - 1:
                    put("final.f32", shard.field())
                    put("arrival.f32", shard.arrival())
            except Exception as exc:
                error = exc
            _agree(error, group, f"frame {k}")
        residual = solver.residual()
        steps = solver.steps
    finally:
        for fd in fds.values():
            os.close(fd)
        if shard is not None and hasattr(shard, "close"):
            shard.close()
    dist.barrier(group)
    meta = {
        "schema": SCHEMA,
        "status": "complete",
        "backend": "b200_cuda_vp_shards",
        "local_precision": local_precision,
        "config": config_dict(config),
        "physics": physics_signature(config),
        "grid": grid.to_dict(),
        "shape": list(grid.shape),
        "state_order": ["x", "y", "psi", "vP", "vE"],
        "axis_order": ["vP", "vE", "psi", "y", "x"],
        "axes": [a.tolist() for a in grid.axes(config)],
        "horizon": horizon,
        "output_dt": output_dt,
        "times": times.tolist(),
        "order": order,
        "cfl": cfl,
        "history_saved": bool(history),
        "dtype": "float32",
        "target": "physical_capture_only",
        "capture_rule": config.capture_rule,
        "avoid": None,
        "tube_projection": "min over every internal update",
        "position_boundary": "one-sided linear extrapolation; outside queries unresolved",
        "speed_boundary": "acceleration restricted to inward or zero at speed limits",
        "heading_boundary": "periodic",
        "cfl_dt_limit": solver.cfl_dt_limit,
        "internal_steps": steps,
        "frames": len(times),
        "last_step_residual": residual,
        "vp_shards": [list(r) for r in ranges],
        "update_seconds": update,
        "total_wall_seconds": time.perf_counter() - started,
    }
    if rank == 0:
        (output / "meta.json").write_text(json.dumps(meta, indent=2) + "\n")
    dist.barrier(group)
    return meta
