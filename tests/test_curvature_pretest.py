"""The curvature sweep's cheap rejection never skips a triplet that acts.

lanes_test (tangle_b200/csrc/kernels.cu) rules a triplet out, before any
IEEE square root, when (u . v) * rsqrtf(|u|^2) * rsqrtf(|v|^2) exceeds a
rough limit cosine by more than 1e-5. The rough limit is the exact path's
formula, 1 - 2 h^2 with h = 0.25 kappa (|u| + |v|), on lengths |u|^2 *
rsqrtf(|u|^2). The exact path (kernels.rs:1165-1322) projects only when
its cosine, from unit vectors made with IEEE divisions, is below its limit
cosine from correctly rounded square roots, with h < 1. The rejection is
exact if rough and exact cosine differ by less than 1e-6 and rough and
exact limit by less than 2e-6 wherever h < 1. rsqrtf is specified to
2 ulp; this models it as the correctly rounded reciprocal square root
moved 2 ulp either way, restates everything in f32 in the kernel's order
of operations, and checks both bounds on random edge pairs: crossed,
nearly parallel and nearly antiparallel, with lengths from 1e-6 to 1e-3 m
(the cheap test needs |u|^2 and |v|^2 above 1e-12), length ratios up to
1e4, and curvature limits that put h anywhere in (0, 1).
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


def rsqrt_models(x):
    """rsqrtf(x) modelled at -2, 0 and +2 ulp of the correctly rounded value."""
    r = (1.0 / np.sqrt(x.astype(np.float64))).astype(f32)
    ulp = (np.nextafter(r, np.inf) - r).astype(f32)
    return [(r + f32(k) * ulp).astype(f32) for k in (-2, 0, 2)]


def cheap_cosines(u, v):
    """(u . v) * (rsqrtf(uu) * rsqrtf(vv)) over every pairing of the models."""
    d = dot(u, v)
    return [(d * (ru * rv).astype(f32)).astype(f32)
            for ru in rsqrt_models(dot(u, u)) for rv in rsqrt_models(dot(v, v))]


def limit_cosine(kappa, lu, lv):
    """1 - 2 h^2 with h = 0.25 kappa (lu + lv), in the kernel's f32 order."""
    h = ((f32(0.25) * kappa).astype(f32) * (lu + lv).astype(f32)).astype(f32)
    return (f32(1.0) - ((f32(2.0) * h).astype(f32) * h).astype(f32)).astype(f32), h


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


def test_rough_limit_cosine_stays_within_a_fifth_of_the_margin():
    rng = np.random.default_rng(11)
    n = 400_000
    lu64 = 10.0 ** rng.uniform(-6, -3, size=n)
    lv64 = lu64 * 10.0 ** rng.uniform(-2, 2, size=n)
    lv64 = np.clip(lv64, 1.0e-6, None)
    a = unit(rng.normal(size=(n, 3)))
    b = unit(rng.normal(size=(n, 3)))
    u = (a * lu64[:, None]).astype(f32)
    v = (b * lv64[:, None]).astype(f32)
    uu, vv = dot(u, u), dot(v, v)
    keep = (uu > f32(1.0e-12)) & (vv > f32(1.0e-12))
    u, v, uu, vv = u[keep], v[keep], uu[keep], vv[keep]
    lu, lv = np.sqrt(uu).astype(f32), np.sqrt(vv).astype(f32)  # correctly rounded, as sqrtf
    h_target = rng.uniform(0.0, 1.0, size=lu.size)
    kappa = (4.0 * h_target / (lu.astype(np.float64) + lv.astype(np.float64))).astype(f32)
    exact, h = limit_cosine(kappa, lu, lv)
    acting = h < f32(1.0)  # the exact path gives up at h >= 1
    worst = 0.0
    for ru in rsqrt_models(uu):
        for rv in rsqrt_models(vv):
            rough, _ = limit_cosine(kappa, (uu * ru).astype(f32), (vv * rv).astype(f32))
            worst = max(worst, float(np.abs(rough.astype(np.float64) - exact)[acting].max()))
    assert worst <= 2.0e-6, worst
