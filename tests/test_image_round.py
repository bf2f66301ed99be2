"""The minimum image's fast path rounds exactly as the division does.

image_round (tangle_b200/csrc/common.cuh) replaces roundf(x / L), the image
count of a periodic axis, by roundf(x * (1 / L)) except where the product
lies within 1e-3 of a half-integer or beyond 4096 box lengths. Its
argument: both quotients lie within 7.4e-4 of the product there, and
rounding to the nearest integer only changes at half-integers. This
restates the fast path in f32 and requires the bits of roundf(x / L),
signed zeros included, on random separations: uniform, near every
half-integer and integer multiple of L, tiny, huge and negative.
"""

import numpy as np

f32 = np.float32


def roundf(v):
    """C roundf (halves away from zero), exact through f64."""
    v64 = v.astype(np.float64)
    return np.copysign(np.floor(np.abs(v64) + 0.5), v64).astype(f32)


def image_round(x, length, inv_length):
    q = (x * inv_length).astype(f32)
    aq = np.abs(q)
    fraction = (aq - np.floor(aq)).astype(f32)
    fast = (aq < f32(4096.0)) & (np.abs((fraction - f32(0.5)).astype(f32)) > f32(1.0e-3))
    slow = roundf((x / length).astype(f32))
    out = np.where(fast, roundf(q), slow)
    return np.where(aq < f32(0.499), np.copysign(f32(0.0), q), out).astype(f32)


def samples(rng, length, n):
    k = rng.integers(-5000, 5000, size=n).astype(np.float64)
    half = (k + 0.5) * float(length) * (1.0 + rng.normal(size=n) * 1e-6)
    whole = k * float(length) * (1.0 + rng.normal(size=n) * 1e-6)
    uniform = rng.uniform(-4.0, 4.0, size=n) * float(length)
    tiny = rng.normal(size=n) * float(length) * 1e-6
    huge = rng.uniform(-1e5, 1e5, size=n) * float(length)
    x = np.concatenate([half, whole, uniform, tiny, huge, -half, [0.0, -0.0]]).astype(f32)
    return x


def test_fast_image_count_matches_division():
    rng = np.random.default_rng(3)
    for length in [f32(2.0e-3), f32(3.0e-4), f32(1.0), f32(7.0), f32(1.234567e-5)] + \
            [f32(v) for v in 10.0 ** rng.uniform(-6, 2, size=20)]:
        inv_length = (f32(1.0) / length).astype(f32)
        x = samples(rng, length, 50_000)
        got = image_round(x, length, inv_length)
        want = roundf((x / length).astype(f32))
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), length
