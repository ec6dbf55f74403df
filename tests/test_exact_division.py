"""The exact stage divides by its grid spacings h and h*h through their
reciprocals rounded to nearest and one FMA correction (Markstein's
correction theorem; csrc/relative5d_exact.cuh, div_const).  The same
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
