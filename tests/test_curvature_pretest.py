"""The curvature sweep's cheap rejection never skips a triplet that acts.

lanes_test (tangle_b200/csrc/kernels.cu) rules a triplet out when
(u . v) * rsqrtf(|u|^2 |v|^2) exceeds the limit's cosine by more than
1e-5; the exact path (kernels.rs:1165-1322) projects only when its cosine,
from unit vectors made with IEEE divisions, is below the limit's cosine.
The rejection is exact if the two cosines never differ by 1e-5. rsqrtf is
specified to 2 ulp; this models it as the correctly rounded reciprocal
square root moved 2 ulp either way, restates both cosines in f32, and
requires them within 1e-6 (a tenth of the margin) on random edge pairs:
crossed, nearly parallel and nearly antiparallel, with lengths from 1e-7
to 1e-3 m and length ratios up to 1e4.
"""

import numpy as np

from test_contact_filters import dot, unit

f32 = np.float32


def exact_cosine(u, v):
    lu = np.sqrt(dot(u, u)).astype(f32)
    lv = np.sqrt(dot(v, v)).astype(f32)
    un = (u / lu[:, None]).astype(f32)
    vn = (v / lv[:, None]).astype(f32)
    return np.clip(dot(un, vn), f32(-1.0), f32(1.0)).astype(f32)


def cheap_cosines(u, v):
    """The rsqrt cosine with rsqrtf at -2, 0 and +2 ulp of the exact value."""
    uv = (dot(u, u) * dot(v, v)).astype(f32)
    r = (1.0 / np.sqrt(uv.astype(np.float64))).astype(f32)
    ulp = (np.nextafter(r, np.inf) - r).astype(f32)
    d = dot(u, v)
    return [(d * (r + f32(k) * ulp).astype(f32)).astype(f32) for k in (-2, 0, 2)]


def test_cheap_cosine_stays_within_a_tenth_of_the_margin():
    rng = np.random.default_rng(9)
    n = 600_000
    a = unit(rng.normal(size=(n, 3)))
    b = unit(rng.normal(size=(n, 3)))
    kind = rng.integers(0, 3, size=n)
    tilt = unit(np.cross(a, rng.normal(size=(n, 3))))
    angle = 10.0 ** rng.uniform(-4, -1, size=n)[:, None]
    b = np.where((kind == 1)[:, None], unit(a * np.cos(angle) + tilt * np.sin(angle)), b)
    b = np.where((kind == 2)[:, None], unit(-a * np.cos(angle) + tilt * np.sin(angle)), b)
    lu = 10.0 ** rng.uniform(-7, -3, size=n)
    lv = lu * 10.0 ** rng.uniform(-2, 2, size=n)
    u = (a * lu[:, None]).astype(f32)
    v = (b * lv[:, None]).astype(f32)
    exact = exact_cosine(u, v)
    worst = max(float(np.abs(c.astype(np.float64) - exact).max()) for c in cheap_cosines(u, v))
    assert worst <= 1.0e-6, worst
