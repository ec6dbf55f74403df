"""The CPU oracle against the reference's own outputs (golden vectors made by
the reference executables, and the executables themselves when built)."""

import ctypes
import shutil

import numpy as np
import pytest

from tests import oracle_lib
from tests.helpers import A3, CONFIG1_GRID, bits, relative_goldens, world_goldens

RELATIVE = relative_goldens()
WORLD = world_goldens()


@pytest.mark.parametrize("name", sorted(RELATIVE))
def test_relative_oracle_reproduces_reference_golden_bitwise(oracle, name):
    case = RELATIVE[name]
    cfg = oracle.rel_cfg(case["config"], case["grid"], order=case["order"])
    assert oracle.rel_cfl_limit(cfg) == pytest.approx(case["cfl_dt_limit"],
                                                      rel=1e-13)
    frames, arrival, steps = oracle.rel_solve_f32(cfg, case["horizon"],
                                                  case["output_dt"])
    assert steps == case["internal_steps"]
    np.testing.assert_array_equal(bits(frames), bits(case["frames"]).reshape(
        frames.shape))
    np.testing.assert_array_equal(bits(arrival), bits(case["arrival"]).ravel())


@pytest.mark.parametrize("name", sorted(WORLD))
def test_world_oracle_reproduces_reference_golden_bitwise(oracle, name):
    z = WORLD[name]
    n, nh, np_, ne = map(int, z["grid"])
    r, pmin, pmax, pa, pk, emin, emax, ea, ek = map(float, z["physics"])
    cfg = oracle_lib.W8Cfg(n, nh, np_, ne, int(z["order"]), int(z["linear"]), 1,
                           float(z["extent"]), float(z["arena"]), r, pmin, pmax,
                           emin, emax, pa, ea, pk, ek, 0.8)
    a, arrival = oracle.w8_init_square(cfg)
    b = np.zeros_like(a)
    maxdt = oracle.w8_dt_limit(cfg)
    horizon, odt = float(z["horizon"]), float(z["output_dt"])
    times = np.unique(np.minimum(np.arange(int(np.ceil(horizon / odt)) + 1) * odt,
                                 horizon))
    tau, steps = 0.0, 0
    for goal in times[1:]:
        while tau < goal - 1e-10:
            dt = min(maxdt, goal - tau)
            if int(z["order"]) == 1:
                oracle.w8_stage(cfg, a, b, None, arrival, dt, tau)
                a, b = b, a
            else:
                oracle.w8_stage(cfg, a, b, None, arrival, dt, tau)
                oracle.w8_stage(cfg, b, a, a, arrival, dt, tau)
            tau += dt
            steps += 1
    assert steps == int(z["internal_steps"])
    np.testing.assert_array_equal(bits(a), bits(z["final"]).ravel())
    np.testing.assert_array_equal(bits(arrival), bits(z["arrival"]).ravel())


@pytest.mark.skipif(not oracle_lib.REF_RELATIVE.exists(),
                    reason="reference executable not built (make -C oracle ref)")
@pytest.mark.parametrize("order", [1, 2])
def test_relative_oracle_matches_reference_executable_on_readme_grid(oracle, order):
    folder, timing = oracle_lib.run_reference_relative(
        A3, CONFIG1_GRID, horizon=0.2, output_dt=0.1, order=order, threads=4)
    try:
        ref = np.fromfile(folder / "fields.f32", np.float32).reshape(3, -1)
        ref_arrival = np.fromfile(folder / "arrival.f32", np.float32)
        cfg = oracle.rel_cfg(A3, CONFIG1_GRID, order=order)
        frames, arrival, steps = oracle.rel_solve_f32(cfg, 0.2, 0.1)
        assert steps == timing["internal_steps"]
        np.testing.assert_array_equal(bits(frames), bits(ref))
        np.testing.assert_array_equal(bits(arrival), bits(ref_arrival))
    finally:
        shutil.rmtree(folder)


def test_fp64_oracle_stays_close_to_float_storage(oracle):
    cfg = oracle.rel_cfg(A3, CONFIG1_GRID)
    frames, _, _ = oracle.rel_solve_f32(cfg, 0.2, 0.1)
    final64, steps = oracle.rel_solve_f64(cfg, 0.2, 0.1)
    assert steps == 18
    err = np.abs(frames[-1].astype(np.float64) - final64)
    # Float storage flips a few ENO stencil choices (|D2_left| vs |D2_centre|
    # ties) at the position-grid corners: rare cells differ by ~1e-4, the
    # bulk by float rounding.
    assert 0 < err.max() < 1e-3
    assert np.quantile(err, 0.999) < 2e-5
    assert err.mean() < 1e-6


def test_tube_is_monotone_and_capture_disk_fixed(oracle):
    cfg = oracle.rel_cfg(A3, CONFIG1_GRID)
    frames, arrival, _ = oracle.rel_solve_f32(cfg, 0.2, 0.1)
    assert np.all(np.diff(frames, axis=0) <= 0)
    inside = frames[0] <= 0
    assert np.all(arrival[inside] == 0)
    assert np.all(np.isnan(arrival[frames[-1] > 0]))


def test_rectangle_contact_known_answers(oracle):
    # tests/test_contact_game.py:21-42 of the reference (default bodies
    # 0.8 x 0.5 and 0.4 x 0.25): exact zeros at contact.
    pb, eb = (0.8, 0.5), (0.4, 0.25)
    p = [0.0, 0.0, 0.0]
    assert oracle.rect_separation(p, [0.6, 0, 0], pb, eb) == pytest.approx(0, abs=1e-15)
    assert oracle.rect_separation(p, [0, 0.375, 0], pb, eb) == pytest.approx(0, abs=1e-15)
    assert oracle.rect_separation(p, [0, 0.5, 0], pb, eb) > 0
    assert oracle.rect_separation(p, [0, 0.5, np.pi / 2], pb, eb) > 0
    assert oracle.rect_separation(p, [0, 0.45, np.pi / 2], pb, eb) == pytest.approx(0, abs=1e-15)
    theta = 0.73
    rot = lambda s: [np.cos(theta) * s[0] - np.sin(theta) * s[1],
                     np.sin(theta) * s[0] + np.cos(theta) * s[1], s[2] + theta]
    assert oracle.rect_separation(rot(p), rot([0, 0.45, np.pi / 2]), pb, eb) == \
        pytest.approx(0, abs=1e-15)


def _w8_rk2_pair(oracle, cfg, a32, steps):
    """`steps` RK2 steps of the float32 stage and of the double stage from the
    same float32 field."""
    a64 = a32.astype(np.float64)
    b32, b64 = np.zeros_like(a32), np.zeros_like(a64)
    dt = oracle.w8_dt_limit(cfg)
    for _ in range(steps):
        assert oracle.w8_stage(cfg, a32, b32, None, None, dt, 0.0) == 0
        assert oracle.w8_stage(cfg, b32, a32, a32, None, dt, 0.0) == 0
        assert oracle.w8_stage_f64(cfg, a64, b64, None, dt) == 0
        assert oracle.w8_stage_f64(cfg, b64, a64, a64, dt) == 0
    return a32, a64


def test_world_fp64_stage_tracks_the_float_stage(oracle):
    """The double-precision 8D stage (the rounding-free yardstick for float32
    variants) against the reference-order float32 stage: float rounding in
    the bulk, rare ENO2 choices flipped at exact ties of the contact field."""
    from pursuit_evasion_b200.reversible.world_dp import WorldGrid

    grid = WorldGrid(5, 4, 3, 3, 3.0)
    p, e = A3.pursuer, A3.evader
    cfg = oracle_lib.W8Cfg(grid.positions, grid.headings, grid.p_speeds,
                           grid.e_speeds, 2, 1, 0, grid.extent,
                           A3.arena_half_width, A3.capture_radius,
                           p.speed_min, p.speed_max, e.speed_min, e.speed_max,
                           p.acceleration, e.acceleration, p.max_curvature,
                           e.max_curvature, 0.8)
    a32, _ = oracle.w8_init_contact(cfg, (0.5, 0.3), (0.5, 0.3))
    f32, f64 = _w8_rk2_pair(oracle, cfg, a32, 5)
    err = np.abs(f32.astype(np.float64) - f64)
    # Measured after 5 steps: mean 1.2e-6, 0.21 % of the cells beyond
    # 2e-5 + 2e-6|v|, max 2.7e-3 -- the reference's own float32 noise.
    assert 0 < err.mean() < 5e-6
    assert np.mean(err > 2e-5 + 2e-6 * np.abs(f64)) < 1e-2
    assert err.max() < 1e-2


SQUARE = __import__("tests.helpers", fromlist=["square_goldens"]).square_goldens()


@pytest.mark.parametrize("name", sorted(SQUARE))
def test_square_oracle_reproduces_reference_golden_bitwise(oracle, name):
    """The 6D square-game restatement (oracle/square6d.c) equals the
    reference executable native_square.cpp bit for bit: every frame, the
    arrival times and the step count."""
    import json

    z = np.load(SQUARE[name])
    options = json.loads(str(z["options"]))
    cfg = oracle.s6_cfg(options)
    # native_timing.json prints the bound with 12 significant digits
    assert oracle.lib.po_s6_dt_limit(ctypes.addressof(cfg)) == pytest.approx(
        float(z["max_internal_dt"]), rel=1e-11)
    frames, arrival, steps = oracle.s6_solve(cfg, options["horizon"], options["output-dt"])
    assert steps == int(z["internal_steps"])
    np.testing.assert_array_equal(bits(frames.reshape(z["fields"].shape)), bits(z["fields"]))
    np.testing.assert_array_equal(bits(arrival), bits(z["arrival"]))
    np.testing.assert_array_equal(bits(frames[-1]), bits(z["final"]))
