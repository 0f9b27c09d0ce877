"""The 6-byte mixed storage format (grg_b200.h, GRG_B200_MIXED), restated in NumPy: FP32 value
rounded to nearest plus a 16-bit correction in units of 2^(e(hi) - 38).  Checks the format's
claims on CPU: the correction always fits in int16 (FP32 rounding ties included), stored
values are within 2^-39 relative, integers below 2^39 round-trip exactly."""

from __future__ import annotations

import numpy as np


def mx_round(v: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    v = np.asarray(v, dtype=np.float64)
    hi = v.astype(np.float32)  # round to nearest, ties to even
    e = ((hi.view(np.uint32) >> 23) & 0xFF).astype(np.int64)
    e = np.maximum(e, 1)
    unit = np.ldexp(1.0, e - 165)
    r = v - hi.astype(np.float64)
    q = np.rint(r / unit)
    return hi, q, hi.astype(np.float64) + q * unit


def test_correction_fits_and_rounding_bound():
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.standard_normal(200_000) * 10.0 ** rng.integers(-30, 30, 200_000),
                        rng.integers(-(2**40), 2**40, 100_000).astype(np.float64)])
    hi, q, back = mx_round(v)
    assert np.all(np.abs(q) <= 2**14)
    assert np.all(np.abs(back - v) <= np.abs(hi.astype(np.float64)) * 2.0**-39)


def test_integers_and_ties_are_exact():
    # every odd integer in [2^24, 2^25) lies exactly halfway between two FP32 values
    odd = np.arange(2**24 + 1, 2**24 + 20_001, 2, dtype=np.float64)
    big = np.random.default_rng(1).integers(-(2**39) + 1, 2**39, 100_000).astype(np.float64)
    for v in (odd, big, -odd):
        hi, q, back = mx_round(v)
        assert np.all(np.abs(q) <= 2**14)
        np.testing.assert_array_equal(back, v)
