"""The reference's own GPU kernels, compiled unchanged and timed on this GPU.

Test and measurement infrastructure, not product code.  The reference ships
its GPU path as CuPy RawKernel source strings: the relative 5D `advance` of
reversible/gpu_relative.py:18-46 (float64 local arithmetic, or float32 via
its textual rewrite `source_code`, :49-64, compiled with --fmad=false,
:134-137) and the 8D `advance` of reversible/gpu_map_game.py:13-75 (float32,
grid sizes substituted as compile-time constants, :152-157).  CuPy is absent
here, so:

    python oracle/ref_gpu.py build   # where the reference tree is mounted:
                                     # its source strings -> nvcc -cubin for
                                     # sm_100a with the reference's options
                                     # -> oracle/_ref/*.cubin (git-ignored)
    python oracle/ref_gpu.py time    # on a B200: load the cubins with the
                                     # CUDA driver API and launch them with
                                     # the reference's argument tuples and
                                     # launch shapes (gpu_relative.py:327-338,
                                     # gpu_map_game.py:208-258)

`time` prints one JSON line per kernel: ms per stage launch from CUDA
events on the launching stream, cells per second and the fraction of the
measured HBM copy bandwidth at the algorithmic 8 / 12 bytes per cell of
the two RK2 stages.  Field values are a capture-distance field; the
kernels' cost does not depend on them.
"""

from __future__ import annotations

import ctypes
import json
import math
import os
from pathlib import Path
import subprocess
import sys
import tempfile

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
REFERENCE = Path(os.environ.get("PE_REFERENCE_ROOT", "/root/reference"))

# the 89M-cell relative grid and the 8D contact grid of the bench
REL_GRID = dict(positions=65, headings=48, p_speeds=21, e_speeds=21, extent=8.0)
W8_GRID = dict(positions=11, headings=9, p_speeds=7, e_speeds=7, extent=3.0)
# reversible_free_a3 (configs/reversible_free_a3.json)
A3 = dict(p_min=-1.0, p_max=2.0, e_min=-0.5, e_max=1.0, ap=3.0, ae=3.0, kp=1.0, ke=2.0,
          radius=0.3)


def cubin(name):
    return OUT / f"{name}.cubin"


def build():
    sys.path.insert(0, str(REFERENCE / "src"))
    from pursuit_evasion.reversible import gpu_map_game, gpu_relative

    g = W8_GRID
    sources = {
        "ref_relative_f32": (gpu_relative.source_code("float32"), ["--fmad=false"]),
        "ref_relative_f64": (gpu_relative.source_code("float64"), ["--fmad=false"]),
        "ref_world8d_11_9_7_7": (
            gpu_map_game.CUDA.replace("@NX@", str(g["positions"]))
            .replace("@NH@", str(g["headings"])).replace("@NV@", str(g["p_speeds"]))
            .replace("@NE@", str(g["e_speeds"])), []),
    }
    OUT.mkdir(exist_ok=True)
    nvcc = "/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else "nvcc"
    with tempfile.TemporaryDirectory() as tmp:
        for name, (text, options) in sources.items():
            src = Path(tmp) / f"{name}.cu"
            src.write_text(text)
            subprocess.run([nvcc, "-cubin", "-arch=sm_100a", "--std=c++17", *options,
                            "-o", str(cubin(name)), str(src)], check=True)
    print("built", ", ".join(sorted(sources)))


class Module:
    """A cubin loaded into the current (primary) context."""

    def __init__(self, path):
        from cuda.bindings import driver as cu

        self.cu = cu
        err, self.mod = cu.cuModuleLoadData(Path(path).read_bytes())
        self._check(err)

    def _check(self, err):
        if int(err) != 0:
            raise RuntimeError(f"CUDA driver error {int(err)}")

    def launch(self, name, grid, block, args, stream):
        cu = self.cu
        err, fn = cu.cuModuleGetFunction(self.mod, name.encode())
        self._check(err)
        values = tuple(v for v, _ in args)
        types = tuple(t for _, t in args)
        (err,) = cu.cuLaunchKernel(fn, grid, 1, 1, block, 1, 1, 0, cu.CUstream(stream),
                                   (values, types), 0)
        self._check(err)


def hbm_peak():
    path = HERE.parent / "MEASURED_PEAKS.json"
    if path.exists():
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def time_relative(precision, steps=10):
    import numpy as np
    import torch

    g = REL_GRID
    n, h, nv, ne = g["positions"], g["headings"], g["p_speeds"], g["e_speeds"]
    N = n * n * h * nv * ne
    real_t = torch.float32 if precision == "float32" else torch.float64
    real_c = ctypes.c_float if precision == "float32" else ctypes.c_double
    dev = torch.device("cuda", 0)
    x = torch.linspace(-g["extent"], g["extent"], n, dtype=torch.float64)
    plane = (torch.hypot(x[None, :], x[:, None]) - A3["radius"]).float()
    a = plane.reshape(-1).to(dev).repeat(N // (n * n))
    b = torch.empty_like(a)
    arrival = torch.full_like(a, float("nan"))
    angles = [-math.pi + i * 2 * math.pi / h for i in range(h)]
    sn = torch.tensor([math.sin(q) for q in angles], dtype=real_t, device=dev)
    cs = torch.tensor([math.cos(q) for q in angles], dtype=real_t, device=dev)
    mod = Module(cubin(f"ref_relative_{'f32' if precision == 'float32' else 'f64'}"))
    stream = torch.cuda.current_stream(dev)
    P = ctypes.c_void_p
    scalars = [(N, ctypes.c_longlong), (n, ctypes.c_int), (h, ctypes.c_int), (nv, ctypes.c_int),
               (ne, ctypes.c_int)] + [
        (v, real_c) for v in (g["extent"], A3["p_min"], A3["p_max"], A3["e_min"],
                              A3["e_max"], A3["ap"], A3["ae"], A3["kp"], A3["ke"])]
    dt = 3.4e-3
    blocks = (N + 127) // 128

    def stage(src, dst, blend, t):
        args = [(src.data_ptr(), P), (dst.data_ptr(), P), (arrival.data_ptr(), P),
                (sn.data_ptr(), P), (cs.data_ptr(), P), *scalars, (dt, real_c), (t, real_c),
                (2, ctypes.c_int), (blend, ctypes.c_int)]
        mod.launch("advance", blocks, 128, args, stream.cuda_stream)

    for k in range(2):  # warm-up
        stage(a, b, 0, k * dt)
        stage(b, a, 1, k * dt)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ms = [0.0, 0.0]
    for k in range(steps):
        ev[0].record(stream)
        stage(a, b, 0, k * dt)
        ev[1].record(stream)
        stage(b, a, 1, k * dt)
        ev[2].record(stream)
        torch.cuda.synchronize()
        ms[0] += ev[0].elapsed_time(ev[1])
        ms[1] += ev[1].elapsed_time(ev[2])
    peak, kind = hbm_peak()
    s1, s2 = ms[0] / steps, ms[1] / steps
    gbs = (8 * N / (s1 / 1e3) + 12 * N / (s2 / 1e3)) / 2 / 1e9
    return {"kernel": f"reference gpu_relative.advance ({precision} local)",
            "grid": "RelativeGrid(65,48,21,21,8.0)", "cells": N,
            "launch": "(N+127)//128 blocks of 128 threads (gpu_relative.py:327-338)",
            "ms_stage1": s1, "ms_stage2": s2,
            "cell_backups_per_s": 2 * N / ((s1 + s2) / 1e3),
            "hbm_frac": ((8 + 12) * N / ((s1 + s2) / 1e3) / 1e9) / peak,
            "peak_gbs": peak, "peak_kind": kind, "steps_timed": steps, "avg_stage_gbs": gbs}


def time_world8d(steps=10):
    import torch

    g = W8_GRID
    n, h, nv, ne = g["positions"], g["headings"], g["p_speeds"], g["e_speeds"]
    N = n ** 4 * h * h * nv * ne
    dev = torch.device("cuda", 0)
    f32 = torch.float32
    a = torch.empty(N, dtype=f32, device=dev)
    b = torch.empty_like(a)
    arrival = torch.empty_like(a)
    free = torch.full((n * n * h,), 1e30, dtype=f32, device=dev)  # no obstacles
    angles = [-math.pi + i * 2 * math.pi / h for i in range(h)]
    sn = torch.tensor([math.sin(q) for q in angles], dtype=f32, device=dev)
    cs = torch.tensor([math.cos(q) for q in angles], dtype=f32, device=dev)
    mod = Module(cubin("ref_world8d_11_9_7_7"))
    stream = torch.cuda.current_stream(dev)
    P, F = ctypes.c_void_p, ctypes.c_float
    blocks = (N + 255) // 256
    mod.launch("init", blocks, 256,
               [(a.data_ptr(), P), (arrival.data_ptr(), P), (free.data_ptr(), P),
                (free.data_ptr(), P), (N, ctypes.c_longlong), (g["extent"], F),
                (A3["radius"], F)], stream.cuda_stream)
    base = [(arrival.data_ptr(), P), (free.data_ptr(), P), (sn.data_ptr(), P),
            (cs.data_ptr(), P), (N, ctypes.c_longlong)] + [
        (v, F) for v in (g["extent"], A3["p_min"], A3["p_max"], A3["e_min"], A3["e_max"],
                         A3["ap"], A3["ae"], A3["kp"], A3["ke"])]
    dt = 1e-2

    def stage(src, dst, blend, t):
        mod.launch("advance", blocks, 256,
                   [(src.data_ptr(), P), (dst.data_ptr(), P), *base, (dt, F), (t, F),
                    (2, ctypes.c_int), (blend, ctypes.c_int)], stream.cuda_stream)

    for k in range(2):
        stage(a, b, 0, k * dt)
        stage(b, a, 1, k * dt)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(steps):
        stage(a, b, 0, k * dt)
        stage(b, a, 1, k * dt)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    peak, kind = hbm_peak()
    return {"kernel": "reference gpu_map_game.advance (float32, obstacle-free clearance)",
            "grid": "WorldGrid(11,9,7,7,3.0)", "cells": N,
            "launch": "(N+255)//256 blocks of 256 threads (gpu_map_game.py:208-258)",
            "ms_per_rk2_step": ms, "cell_backups_per_s": 2 * N / (ms / 1e3),
            "hbm_frac": (20 * N / (ms / 1e3) / 1e9) / peak, "peak_gbs": peak,
            "peak_kind": kind, "steps_timed": steps}


def main():
    mode = sys.argv[1] if len(sys.argv) > 1 else "time"
    if mode == "build":
        build()
        return
    import torch

    torch.cuda.init()
    torch.cuda.synchronize()
    for fn in (lambda: time_relative("float32"), lambda: time_relative("float64"),
               time_world8d):
        print(json.dumps(fn()), flush=True)


if __name__ == "__main__":
    main()
