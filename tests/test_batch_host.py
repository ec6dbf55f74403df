"""Host side of the batched solver: the seeded solve set, the autotuner's
buckets and candidates, and the C ABI's option checks (no GPU needed)."""

import ctypes

import numpy as np
import pytest

from pursuit_evasion_b200 import _native
from pursuit_evasion_b200.batch import autotune, describe, draw_batch
from pursuit_evasion_b200.reversible.relative_solver import _params


def test_draw_batch_is_seeded_and_within_ranges():
    a, b = draw_batch(11), draw_batch(11)
    assert describe(a) == describe(b)
    assert describe(a) != describe(draw_batch(12))
    assert len(a) == 256
    t = describe(a)
    pos = np.array([r["positions"] for r in t])
    assert pos.min() >= 17 and pos.max() <= 49
    hd = np.array([r["headings"] for r in t])
    assert hd.min() >= 12 and hd.max() <= 36
    for key in ("p_speeds", "e_speeds"):
        v = np.array([r[key] for r in t])
        assert v.min() >= 7 and v.max() <= 15
    for key, lo, hi in (("p_acceleration", 1.5, 4), ("e_acceleration", 1.5, 4),
                        ("capture_radius", 0.3, 0.8), ("horizon", 0.5, 2)):
        v = np.array([r[key] for r in t])
        assert v.min() >= lo and v.max() <= hi


def test_buckets_and_candidates():
    assert autotune.bucket_of(17) == "17-24"
    assert autotune.bucket_of(33) == "33-40"
    assert autotune.bucket_of(49) == "41-49"
    assert autotune.bucket_of(65) == "other"
    for n in (17, 24, 33, 49):
        assert all(r * n >= 256 and r <= n for r in autotune.candidates(n))
        # tiled float32 kernel: at most one 4-cell chunk per thread of 256
        tiled = autotune.candidates(n, "float32")
        assert tiled and all(1 <= r <= n and r * ((n + 3) // 4) <= 256 for r in tiled)
    assert autotune.candidates(17) == [16]
    assert autotune.candidates(49, "float32")[-1] == 19
    # a bucket of 34- to 40-wide grids: every candidate fits a 40-wide CTA
    assert autotune.candidates(34, "float32", 40)[-1] == 25
    assert max(autotune.candidates(34, "float32", 40)) * 10 <= 256


@pytest.mark.parametrize("field, value", [("order", 1), ("precision", _native.PE_LOCAL_F32),
                                          ("positions", 2)])
def test_create_rejects_unsupported_options(field, value):
    lib = _native.library()
    s = draw_batch(1, count=2)
    params = (_native.RelativeParams * 2)(*[
        _params(x.config, x.grid, order=2, cfl=0.8, precision=_native.PE_LOCAL_F64, device=0)
        for x in s])
    setattr(params[1], field, value)
    horizons = (ctypes.c_double * 2)(0.5, 0.5)
    h = ctypes.c_void_p()
    assert lib.pe_batch_create(params, horizons, 2, 0, ctypes.byref(h)) == _native.PE_EINVAL
    assert b"solve 1" in lib.pe_last_error()


def test_create_rejects_bad_horizon():
    lib = _native.library()
    s = draw_batch(1, count=1)
    params = (_native.RelativeParams * 1)(
        _params(s[0].config, s[0].grid, order=2, cfl=0.8, precision=_native.PE_LOCAL_F64,
                device=0))
    for bad in (0.0, -1.0, float("nan")):
        h = ctypes.c_void_p()
        horizons = (ctypes.c_double * 1)(bad)
        assert lib.pe_batch_create(params, horizons, 1, 0, ctypes.byref(h)) == _native.PE_EINVAL
