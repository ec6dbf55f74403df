"""ctypes access to the CPU oracle (oracle/_build/liboracle.so) and to the
reference executables built from the reference sources (oracle/_ref/).

Test infrastructure only: the checker the CUDA path is compared against.
"""

from __future__ import annotations

import ctypes
import json
from pathlib import Path
import subprocess
import tempfile

import numpy as np

REPO = Path(__file__).resolve().parents[1]
ORACLE_DIR = REPO / "oracle"
ORACLE_LIB = ORACLE_DIR / "_build" / "liboracle.so"
REF_RELATIVE = ORACLE_DIR / "_ref" / "relative5d"
REF_WORLD = ORACLE_DIR / "_ref" / "reversible_world8d"


class RelCfg(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("nx", "nh", "nvp", "nve", "order")] + [
        (n, ctypes.c_double)
        for n in ("extent", "radius", "vp_lo", "vp_hi", "ve_lo", "ve_hi",
                  "acc_p", "acc_e", "curv_p", "curv_e", "cfl")
    ]


class W8Cfg(ctypes.Structure):
    _fields_ = [
        (n, ctypes.c_int)
        for n in ("n", "nh", "np", "ne", "order", "linear_speed", "avoid_square")
    ] + [
        (n, ctypes.c_float)
        for n in ("extent", "arena", "radius", "p_lo", "p_hi", "e_lo", "e_hi",
                  "ap", "ae", "kp", "ke")
    ] + [("cfl", ctypes.c_double)]


class S6Cfg(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("n", "nh", "order")] + [
        (n, ctypes.c_float) for n in ("extent", "arena", "radius", "vp", "ve", "wp", "we")
    ] + [("cfl", ctypes.c_double)]


class SLCfg(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("nx", "nh", "nvp", "nve", "mode")] + [
        (n, ctypes.c_double)
        for n in ("extent", "radius", "vp_lo", "vp_hi", "ve_lo", "ve_hi",
                  "acc_p", "acc_e", "curv_p", "curv_e", "dt")
    ]


SL_TUBE, SL_MINTIME = 0, 1

_P = ctypes.c_void_p


def _build():
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


class Oracle:
    def __init__(self, lib):
        self.lib = lib
        sig = {
            "po_rel_cells": (ctypes.c_size_t, [_P]),
            "po_div_const_check": (ctypes.c_longlong, [ctypes.c_double, ctypes.c_longlong,
                                                       ctypes.c_ulonglong]),
            "po_div_const_checkf": (ctypes.c_longlong, [ctypes.c_float, ctypes.c_longlong,
                                                        ctypes.c_ulonglong]),
            "po_rel_cfl_limit": (ctypes.c_double, [_P]),
            "po_rel_init": (None, [_P, _P, _P]),
            "po_rel_init_f64": (None, [_P, _P]),
            "po_rel_stage_f32": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_int, _P]),
            "po_rel_stage_f64": (ctypes.c_int, [_P, _P, _P, ctypes.c_double,
                                                ctypes.c_int]),
            "po_rel_solve_f32": (ctypes.c_int, [_P, ctypes.c_double,
                                                ctypes.c_double, _P, _P, _P]),
            "po_rel_solve_f64": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double,
                                                _P, _P]),
            "po_w8_cells": (ctypes.c_size_t, [_P]),
            "po_w8_dt_limit": (ctypes.c_double, [_P]),
            "po_w8_init_square": (None, [_P, _P, _P]),
            "po_rect_separation": (ctypes.c_double, [ctypes.c_double] * 10),
            "po_w8_init_contact": (None, [_P] + [ctypes.c_double] * 4 + [_P, _P]),
            "po_w8_stage_f64": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_double]),
            "po_s6_cells": (ctypes.c_size_t, [_P]),
            "po_s6_dt_limit": (ctypes.c_double, [_P]),
            "po_s6_init": (None, [_P, _P, _P]),
            "po_s6_stage": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_float,
                                           ctypes.c_double]),
            "po_w8_stage": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_float,
                                           ctypes.c_double]),
            "po_w8_stage_clear": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_float,
                                                 ctypes.c_double, _P]),
            "po_w8_init_map": (None, [_P, _P, _P, _P, _P]),
            "po_sl_integrated_speed": (None, [ctypes.c_double] * 5 + [_P, _P]),
            "po_sl_successor": (None, [_P] + [ctypes.c_double] * 5
                                + [ctypes.c_int, ctypes.c_int, _P]),
            "po_sl_interpolate": (ctypes.c_double, [_P, _P, _P]),
            "po_sl_backup": (ctypes.c_int, [_P, _P, _P, _P, _P]),
            "po_sl_init": (None, [_P, _P]),
            "po_sl_backup_cells": (None, [_P, _P, ctypes.c_size_t, _P, _P, _P, _P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args

    # -- relative 5D ---------------------------------------------------------
    @staticmethod
    def rel_cfg(config, grid, order=2, cfl=0.8):
        p, e = config.pursuer, config.evader
        return RelCfg(grid.positions, grid.headings, grid.p_speeds,
                      grid.e_speeds, order, grid.extent, config.capture_radius,
                      p.speed_min, p.speed_max, e.speed_min, e.speed_max,
                      p.acceleration, e.acceleration, p.max_curvature,
                      e.max_curvature, cfl)

    def rel_cfl_limit(self, cfg):
        return self.lib.po_rel_cfl_limit(ctypes.addressof(cfg))

    def rel_solve_f32(self, cfg, horizon, output_dt):
        """Frames [T, N] and arrival of the reference executable's solve."""
        n = self.lib.po_rel_cells(ctypes.addressof(cfg))
        count = int(np.ceil(horizon / output_dt - 1e-10)) + 1
        frames = np.zeros((count, n), np.float32)
        arrival = np.zeros(n, np.float32)
        steps = ctypes.c_long()
        rc = self.lib.po_rel_solve_f32(ctypes.addressof(cfg), horizon, output_dt,
                                       frames.ctypes.data, arrival.ctypes.data,
                                       ctypes.addressof(steps))
        assert rc == 0, rc
        return frames, arrival, steps.value

    def rel_solve_f64(self, cfg, horizon, output_dt):
        """Final field of the same step sequence with double storage."""
        n = self.lib.po_rel_cells(ctypes.addressof(cfg))
        final = np.zeros(n, np.float64)
        steps = ctypes.c_long()
        rc = self.lib.po_rel_solve_f64(ctypes.addressof(cfg), horizon, output_dt,
                                       final.ctypes.data, ctypes.addressof(steps))
        assert rc == 0, rc
        return final, steps.value

    def rel_stage_f32(self, cfg, src, dst, arrival, dt, t, blend):
        inc = ctypes.c_double()
        rc = self.lib.po_rel_stage_f32(ctypes.addressof(cfg), src.ctypes.data,
                                       dst.ctypes.data,
                                       None if arrival is None else arrival.ctypes.data,
                                       dt, t, blend, ctypes.addressof(inc))
        return rc, inc.value

    # -- dense 8D ------------------------------------------------------------
    def w8_cells(self, cfg):
        return self.lib.po_w8_cells(ctypes.addressof(cfg))

    def w8_dt_limit(self, cfg):
        return self.lib.po_w8_dt_limit(ctypes.addressof(cfg))

    def w8_init_square(self, cfg):
        n = self.w8_cells(cfg)
        a = np.zeros(n, np.float32)
        arr = np.zeros(n, np.float32)
        self.lib.po_w8_init_square(ctypes.addressof(cfg), a.ctypes.data,
                                   arr.ctypes.data)
        return a, arr

    def w8_init_contact(self, cfg, p_body, e_body):
        n = self.w8_cells(cfg)
        a = np.zeros(n, np.float32)
        arr = np.zeros(n, np.float32)
        self.lib.po_w8_init_contact(ctypes.addressof(cfg), p_body[0], p_body[1],
                                    e_body[0], e_body[1], a.ctypes.data,
                                    arr.ctypes.data)
        return a, arr

    def w8_init_map(self, cfg, p_clear, e_clear):
        n = self.w8_cells(cfg)
        a = np.zeros(n, np.float32)
        arr = np.zeros(n, np.float32)
        pc = np.ascontiguousarray(p_clear, np.float32)
        ec = np.ascontiguousarray(e_clear, np.float32)
        self.lib.po_w8_init_map(ctypes.addressof(cfg), pc.ctypes.data, ec.ctypes.data,
                                a.ctypes.data, arr.ctypes.data)
        return a, arr

    def w8_stage_clear(self, cfg, src, dst, base, arrival, dt, tau, p_clear):
        pc = np.ascontiguousarray(p_clear, np.float32)
        return self.lib.po_w8_stage_clear(ctypes.addressof(cfg), src.ctypes.data,
                                          dst.ctypes.data,
                                          None if base is None else base.ctypes.data,
                                          None if arrival is None else arrival.ctypes.data,
                                          dt, tau, pc.ctypes.data)

    def w8_stage(self, cfg, src, dst, base, arrival, dt, tau):
        return self.lib.po_w8_stage(ctypes.addressof(cfg), src.ctypes.data,
                                    dst.ctypes.data,
                                    None if base is None else base.ctypes.data,
                                    None if arrival is None else arrival.ctypes.data,
                                    dt, tau)

    def w8_stage_f64(self, cfg, src, dst, base, dt):
        """One stage on float64 fields (no arrival)."""
        for a in (src, dst) + (() if base is None else (base,)):
            assert a.dtype == np.float64 and a.flags.c_contiguous
        return self.lib.po_w8_stage_f64(ctypes.addressof(cfg), src.ctypes.data,
                                        dst.ctypes.data,
                                        None if base is None else base.ctypes.data,
                                        dt)

    # -- legacy 6D square game ---------------------------------------------
    @staticmethod
    def s6_cfg(options):
        """S6Cfg from the reference executable's options (its defaults for the
        missing ones, native_square.cpp:65-80)."""
        o = dict(extent=3.5, arena=3.0, radius=0.3, vp=1.0, ve=0.3, wp=1.0, we=2.0,
                 order=2, cfl=0.8)
        o.update(options)
        return S6Cfg(int(o["positions"]), int(o["headings"]), int(o["order"]),
                     o["extent"], o["arena"], o["radius"], o["vp"], o["ve"], o["wp"],
                     o["we"], o["cfl"])

    def s6_solve(self, cfg, horizon, output_dt):
        """The executable's frame loop (native_square.cpp:185-202): frames,
        final arrival and the number of internal steps."""
        n = self.lib.po_s6_cells(ctypes.addressof(cfg))
        a, b = np.zeros(n, np.float32), np.zeros(n, np.float32)
        arrival = np.zeros(n, np.float32)
        self.lib.po_s6_init(ctypes.addressof(cfg), a.ctypes.data, arrival.ctypes.data)
        frames = [a.copy()]
        maxdt = self.lib.po_s6_dt_limit(ctypes.addressof(cfg))
        tau, steps = 0.0, 0
        for frame in range(1, int(np.ceil(horizon / output_dt - 1e-10)) + 1):
            goal = min(horizon, frame * output_dt)
            while tau < goal - 1e-10:
                dt = np.float32(min(maxdt, goal - tau))
                if cfg.order == 1:
                    self.lib.po_s6_stage(ctypes.addressof(cfg), a.ctypes.data, b.ctypes.data,
                                         None, arrival.ctypes.data, dt, tau)
                    a, b = b, a
                else:
                    self.lib.po_s6_stage(ctypes.addressof(cfg), a.ctypes.data, b.ctypes.data,
                                         None, arrival.ctypes.data, dt, tau)
                    self.lib.po_s6_stage(ctypes.addressof(cfg), b.ctypes.data, a.ctypes.data,
                                         a.ctypes.data, arrival.ctypes.data, dt, tau)
                tau += min(maxdt, goal - tau)
                steps += 1
            frames.append(a.copy())
        return np.array(frames), arrival, steps

    # -- semi-Lagrangian 5D -----------------------------------------------
    @staticmethod
    def sl_cfg(config, grid, dt, mode=SL_TUBE):
        p, e = config.pursuer, config.evader
        return SLCfg(grid.positions, grid.headings, grid.p_speeds, grid.e_speeds,
                     mode, grid.extent, config.capture_radius, p.speed_min,
                     p.speed_max, e.speed_min, e.speed_max, p.acceleration,
                     e.acceleration, p.max_curvature, e.max_curvature, dt)

    def sl_successor(self, cfg, state, up, ue):
        out = np.zeros(5)
        self.lib.po_sl_successor(ctypes.addressof(cfg), *map(float, state), up, ue,
                                 out.ctypes.data)
        return out

    def sl_interpolate(self, cfg, V, state):
        s = np.ascontiguousarray(state, dtype=np.float64)
        return self.lib.po_sl_interpolate(ctypes.addressof(cfg), V.ctypes.data,
                                          s.ctypes.data)

    def sl_init(self, cfg, n):
        V = np.zeros(n)
        self.lib.po_sl_init(ctypes.addressof(cfg), V.ctypes.data)
        return V

    def sl_backup(self, cfg, V, with_policy=False):
        V = np.ascontiguousarray(V, dtype=np.float64)
        out = np.zeros_like(V)
        pp = np.zeros(V.size, np.uint8) if with_policy else None
        pe = np.zeros(V.size, np.uint8) if with_policy else None
        rc = self.lib.po_sl_backup(ctypes.addressof(cfg), V.ctypes.data,
                                   out.ctypes.data,
                                   None if pp is None else pp.ctypes.data,
                                   None if pe is None else pe.ctypes.data)
        assert rc == 0, rc
        return (out, pp, pe) if with_policy else out

    def sl_backup_cells(self, cfg, V, cells):
        """Backup of the listed flat cells only: (values, policy_p, policy_e)."""
        V = np.ascontiguousarray(V, dtype=np.float64)
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        out = np.zeros(len(cells))
        pp = np.zeros(len(cells), np.uint8)
        pe = np.zeros(len(cells), np.uint8)
        self.lib.po_sl_backup_cells(ctypes.addressof(cfg), V.ctypes.data, len(cells),
                                    cells.ctypes.data, out.ctypes.data,
                                    pp.ctypes.data, pe.ctypes.data)
        return out, pp, pe

    def rect_separation(self, p, e, p_body, e_body):
        return self.lib.po_rect_separation(p[0], p[1], p[2], e[0], e[1], e[2],
                                           p_body[0], p_body[1], e_body[0],
                                           e_body[1])


_oracle = None


def load():
    global _oracle
    if _oracle is None:
        if not ORACLE_LIB.exists():
            _build()
        _oracle = Oracle(ctypes.CDLL(str(ORACLE_LIB)))
    return _oracle


def run_reference_relative(config, grid, *, horizon, output_dt, order=2,
                           cfl=0.8, threads=4, history=True):
    """Run the reference executable (built from native_relative.cpp) with the
    argv free_dp.solve would pass (free_dp.py:198-224); returns its output
    folder.  Requires oracle/_ref/relative5d."""
    p, e = config.pursuer, config.evader
    folder = Path(tempfile.mkdtemp(prefix="pe_ref_"))
    options = {
        "positions": grid.positions, "headings": grid.headings,
        "p-speeds": grid.p_speeds, "e-speeds": grid.e_speeds,
        "extent": grid.extent, "radius": config.capture_radius,
        "p-min": p.speed_min, "p-max": p.speed_max,
        "e-min": e.speed_min, "e-max": e.speed_max,
        "p-acceleration": p.acceleration, "e-acceleration": e.acceleration,
        "p-curvature": p.max_curvature, "e-curvature": e.max_curvature,
        "horizon": horizon, "output-dt": output_dt, "order": order, "cfl": cfl,
        "threads": threads, "history": int(history), "output": str(folder),
    }
    cmd = [str(REF_RELATIVE)] + [str(x) for k, v in options.items()
                                 for x in ("--" + k, v)]
    subprocess.run(cmd, check=True, capture_output=True)
    return folder, json.loads((folder / "timing.json").read_text())
