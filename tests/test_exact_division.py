"""The exact stages divide by their grid spacings h and h*h through their
reciprocals rounded to nearest and one FMA correction (Markstein's
correction theorem; csrc/div_rn.cuh, rn::div_const): the relative 5D stage
in double, the 8D and 6D stages in float.  The same
sequence in the host's IEEE double arithmetic (oracle/divcheck.c) must give
a / b in every bit for the spacings of the reference's grids and for random
spacings, over dividends of the kinds the stage divides: differences and
second differences of floats, random doubles over a wide exponent range,
signed zeros and subnormals.  The GPU parity tests check the stage itself
against the reference executable bit for bit."""

import math

import numpy as np


def spacings():
    out = []
    for positions, extent in ((17, 4.0), (33, 8.0), (65, 8.0), (129, 8.0), (49, 4.0)):
        out.append(2 * extent / (positions - 1))
    for headings in (8, 12, 24, 36, 48, 64):
        out.append(2 * math.pi / headings)
    for lo, hi, n in ((-1.0, 2.0, 7), (-1.0, 2.0, 21), (-0.5, 1.0, 21), (-0.5, 1.0, 15)):
        out.append((hi - lo) / (n - 1))
    rng = np.random.default_rng(7)
    out += list(np.ldexp(1.0 + rng.random(12), rng.integers(-8, 6, 12)))
    return out + [h * h for h in out]


def test_division_by_a_spacing_equals_ieee_division(oracle):
    for k, b in enumerate(spacings()):
        assert oracle.lib.po_div_const_check(float(b), 200_000, 1000 + k) == 0, b


def test_float_division_by_a_spacing_equals_ieee_division(oracle):
    f32 = np.float32
    hs = [f32(2 * f32(e)) / f32(n - 1) for n, e in ((11, 3.0), (9, 4.0), (7, 3.0), (17, 3.5))]
    hs += [f32(2 * math.pi / nh) for nh in (9, 8, 16, 5, 4)]
    hs += [f32(3.0) / f32(6), f32(1.5) / f32(6), f32(0.5) / f32(2)]
    rng = np.random.default_rng(11)
    hs += list(np.ldexp(f32(1) + rng.random(12).astype(f32), rng.integers(-8, 4, 12)).astype(f32))
    for k, b in enumerate(hs + [f32(h * h) for h in hs]):
        assert oracle.lib.po_div_const_checkf(float(b), 200_000, 500 + k) == 0, b
