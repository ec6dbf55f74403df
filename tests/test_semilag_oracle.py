"""Pins of the FP64 semi-Lagrangian oracle (no reference 5D semi-Lagrangian
solver exists, so the pieces are pinned one by one):
  * successors against golden vectors produced by the reference's own
    joint_step / relative_state / action_catalogue (tests/golden/
    make_successor_golden.py), and the reference test's known answers of
    integrated_speed (tests/test_reversible_model.py:15-25);
  * interpolation: exact on multilinear fields, periodic in heading;
  * the backup against an independent NumPy brute force of the min-max
    with the tube minimum and the pursuer/evader tie rules."""

from itertools import product

import numpy as np
import pytest

from tests import oracle_lib
from tests.helpers import A3, GOLDEN
from pursuit_evasion_b200.reversible.free_dp import RelativeGrid

SUCC = np.load(GOLDEN / "sl_successors.npz")


def wrap(a):
    return (a + np.pi) % (2 * np.pi) - np.pi


@pytest.mark.parametrize("t", range(3))
def test_successors_match_reference_model(oracle, t):
    dt = float(SUCC["dts"][t])
    cfg = oracle.sl_cfg(A3, RelativeGrid(9, 8, 7, 7, 4.0), dt)
    worst = 0.0
    for i, s in list(enumerate(SUCC["states"]))[::4]:
        for up in range(9):
            for ue in range(9):
                got = oracle.sl_successor(cfg, s, up, ue)
                ref = SUCC["successors"][t, i, up, ue]
                d = got - ref
                d[2] = wrap(d[2])
                worst = max(worst, np.abs(d).max())
    assert worst < 1e-12


def test_integrated_speed_known_answers(oracle):
    import ctypes
    for (v, a, d), (v_ref, d_ref) in zip(SUCC["speed_cases"], SUCC["speed_answers"]):
        vo, do = ctypes.c_double(), ctypes.c_double()
        oracle.lib.po_sl_integrated_speed(v, a, d, -1.0, 2.0, ctypes.addressof(vo),
                                          ctypes.addressof(do))
        assert vo.value == pytest.approx(v_ref, abs=1e-14)
        assert do.value == pytest.approx(d_ref, abs=1e-14)
    vo, do = ctypes.c_double(), ctypes.c_double()
    oracle.lib.po_sl_integrated_speed(1.5, 2.0, 1.0, -1, 2, ctypes.addressof(vo),
                                      ctypes.addressof(do))
    assert (vo.value, do.value) == (2.0, 1.9375)


def test_interpolation_exact_on_multilinear_fields_and_periodic(oracle):
    grid = RelativeGrid(9, 8, 5, 4, 2.0)
    cfg = oracle.sl_cfg(A3, grid, 0.05)
    vp, ve, psi, y, x = np.meshgrid(*grid.axes(A3), indexing="ij")
    field = 1.5 * x - 0.7 * y + 0.3 * vp - 0.4 * ve + 0.2 * x * vp
    field = np.ascontiguousarray(field.ravel())
    rng = np.random.default_rng(3)
    for _ in range(200):
        s = np.array([rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(-4, 4),
                      rng.uniform(-1, 2), rng.uniform(-0.5, 1)])
        expect = 1.5 * s[0] - 0.7 * s[1] + 0.3 * s[3] - 0.4 * s[4] + 0.2 * s[0] * s[3]
        assert oracle.sl_interpolate(cfg, field, s) == pytest.approx(expect, abs=1e-12)
    # linear extrapolation beyond the position box
    s = np.array([2.5, -2.3, 0.0, 0.5, 0.2])
    expect = 1.5 * 2.5 + 0.7 * 2.3 + 0.15 - 0.08 + 0.25
    assert oracle.sl_interpolate(cfg, field, s) == pytest.approx(expect, abs=1e-12)
    # heading periodicity on a heading-dependent field
    field2 = np.ascontiguousarray((np.cos(psi) + 0 * x).ravel())
    a = oracle.sl_interpolate(cfg, field2, np.array([0.1, 0.2, 3.0, 0.0, 0.0]))
    b = oracle.sl_interpolate(cfg, field2, np.array([0.1, 0.2, 3.0 - 2 * np.pi, 0.0, 0.0]))
    assert a == pytest.approx(b, abs=1e-12)


# ---------------------------------------------------------------- brute force
def np_successor(config, s, u, w, dt):
    """Independent NumPy restatement of the held-command relative successor."""
    def speed(v, a, lim):
        target = lim.speed_max if a >= 0 else lim.speed_min
        hit = (target - v) / a if abs(a) > 1e-14 else np.inf
        active = min(dt, max(0.0, hit))
        final = min(max(v + a * dt, lim.speed_min), lim.speed_max)
        return final, v * active + 0.5 * a * active ** 2 + final * (dt - active)

    x, y, psi, vp, ve = s
    vp2, dp = speed(vp, u[0], config.pursuer)
    ve2, de = speed(ve, w[0], config.evader)
    tp, te = u[1] * dp, w[1] * de
    cp_ = dp * np.sinc(tp / (2 * np.pi))
    ce = de * np.sinc(te / (2 * np.pi))
    P = np.array([cp_ * np.cos(tp / 2), cp_ * np.sin(tp / 2)])
    Epos = np.array([x + ce * np.cos(psi + te / 2), y + ce * np.sin(psi + te / 2)])
    d = Epos - P
    return np.array([np.cos(tp) * d[0] + np.sin(tp) * d[1],
                     -np.sin(tp) * d[0] + np.cos(tp) * d[1],
                     wrap(psi + te - tp), vp2, ve2])


def np_interp(grid, config, V, s):
    axes = grid.axes(config)
    vals = [s[3], s[4], s[2], s[1], s[0]]
    js, ws = [], []
    for k, (axis, q) in enumerate(zip(axes, vals)):
        h = axis[1] - axis[0]
        n = len(axis)
        if k == 2:
            f = (q + np.pi) / h
            j = int(np.floor(f))
            ws.append(f - j)
            js.append([j % n, (j + 1) % n])
        else:
            f = (q - axis[0]) / h
            j = min(max(int(np.floor(f)), 0), n - 2)
            ws.append(f - j)
            js.append([j, j + 1])
    total = 0.0
    for bits in product([0, 1], repeat=5):
        w = np.prod([ws[k] if b else 1 - ws[k] for k, b in enumerate(bits)])
        total += w * V[tuple(js[k][b] for k, b in enumerate(bits))]
    return total


E_PREFERENCE = [4, 1, 7, 3, 5, 0, 2, 6, 8]


@pytest.mark.parametrize("mode", [oracle_lib.SL_TUBE, oracle_lib.SL_MINTIME])
def test_backup_matches_bruteforce(oracle, mode):
    grid = RelativeGrid(5, 4, 3, 3, 1.5)
    dt = 0.07
    cfg = oracle.sl_cfg(A3, grid, dt, mode)
    rng = np.random.default_rng(11)
    V = rng.uniform(0, 1, grid.shape) if mode == oracle_lib.SL_MINTIME else \
        rng.normal(size=grid.shape)
    out, pp, pe = oracle.sl_backup(cfg, V.ravel(), with_policy=True)
    P = [(a, k) for a in (-3.0, 0.0, 3.0) for k in (-1.0, 0.0, 1.0)]
    E = [(a, k) for a in (-3.0, 0.0, 3.0) for k in (-2.0, 0.0, 2.0)]
    axes = grid.axes(A3)
    cells = list(np.ndindex(*grid.shape))
    picks = rng.choice(len(cells), size=60, replace=False)
    for idx in [cells[i] for i in picks]:
        iv, ie, ip, iy, ix = idx
        s = np.array([axes[4][ix], axes[3][iy], axes[2][ip], axes[0][iv], axes[1][ie]])
        worst, worst_e = [], []
        for u in P:
            vals = []
            for w in E:
                v = np_interp(grid, A3, V, np_successor(A3, s, u, w, dt))
                if mode == oracle_lib.SL_MINTIME:
                    v = min(max(v, 0.0), 1.0)
                vals.append(v)
            m = max(vals)
            worst.append(m)
            worst_e.append(next(e for e in E_PREFERENCE if vals[e] >= m - 1e-7))
        best = min(worst)
        tied = [u for u in range(9) if worst[u] <= best + 1e-7]
        pick = min(tied, key=lambda u: (abs(u % 3 - 1), abs(u // 3 - 1), u))
        if mode == oracle_lib.SL_TUBE:
            expect = min(best, V[idx])
        else:
            d = np.hypot(s[0], s[1]) - A3.capture_radius
            expect = 0.0 if d <= 0 else (1 - np.exp(-dt)) + np.exp(-dt) * best
        flat = np.ravel_multi_index(idx, grid.shape)
        assert out[flat] == pytest.approx(expect, abs=1e-12)
        assert pp[flat] == pick
        assert pe[flat] == worst_e[pick]
