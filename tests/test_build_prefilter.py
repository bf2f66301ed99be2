"""The Verlet build's sphere pre-test passes every pair the exact test accepts.

rb_build_kernel (tangle_b200/csrc/kernels.cu) tests 32 candidates at a
time against the home segment's bounding sphere (midpoint, half length +
radius), with the threshold (R1 + R2 + skin) x 1.0002 + 1e-6 of the box
edge and the nearest-integer image, and gives only the survivors the
reference's exact test (build_pair: minimum image, midpoint reach, axis
distance within (r1 + r2 + skin) x 1.0001; neighbor.rs:282-359). This
restates both in f32, operation for operation, at the mid-size specimen's
scale in a periodic 2 mm cell: pairs whose axes come within 0.9-1.05 of
the interaction distance, axes from crossed to within 0.005 rad of
parallel, pairs end to end at the interaction distance (where the sphere
bound is tight), both segments unwrapped by up to two box lengths either
way.
Every pair the exact test accepts must pass the sphere test.
"""

import numpy as np

from test_contact_filters import as_f32, distance, dot, unit

f32 = np.float32
LENGTH = f32(2.0e-3)
INV_LENGTH = (f32(1.0) / LENGTH).astype(f32)
SKIN = f32(2.0) * f32(9.5e-6)  # neighbor skin: 2 x the largest radius
SPHERE_EPS = f32(1.0e-6) * LENGTH


def roundf(v):
    v64 = v.astype(np.float64)
    return np.copysign(np.floor(np.abs(v64) + 0.5), v64).astype(f32)


def half_length(p, q):
    d = (q - p).astype(f32)
    return (f32(0.5) * np.sqrt(dot(d, d))).astype(f32)


def exact_build_test(p1, q1, r1, p2, q2, r2):
    """build_pair's geometric tests after the minimum image."""
    image = (f32(0.5) * (((p2 + q2).astype(f32) - p1).astype(f32) - q1).astype(f32)).astype(f32)
    shift = (roundf((image / LENGTH).astype(f32)) * LENGTH).astype(f32)
    moved = np.any(shift != 0.0, axis=1)
    s2, t2 = (p2 - shift).astype(f32), (q2 - shift).astype(f32)
    d1, d2 = (q1 - p1).astype(f32), (t2 - s2).astype(f32)
    interaction = (((r1 + r2).astype(f32) + SKIN).astype(f32) * f32(1.0001)).astype(f32)
    m = (f32(0.5) * (((s2 + t2).astype(f32) - p1).astype(f32) - q1).astype(f32)).astype(f32)
    other_half = np.where(moved, (f32(0.5) * np.sqrt(dot(d2, d2))).astype(f32), half_length(p2, q2))
    reach = ((half_length(p1, q1) + other_half).astype(f32) + interaction).astype(f32)
    near = dot(m, m) <= (reach * reach).astype(f32)
    return near & (distance(p1, d1, s2, d2, False) <= interaction)


def sphere_test(p1, q1, r1, p2, q2, r2):
    c1 = (f32(0.5) * (p1 + q1).astype(f32)).astype(f32)
    c2 = (f32(0.5) * (p2 + q2).astype(f32)).astype(f32)
    w1 = (half_length(p1, q1) + r1).astype(f32)
    w2 = (half_length(p2, q2) + r2).astype(f32)
    d = (c2 - c1).astype(f32)
    d = (d - (np.rint((d * INV_LENGTH).astype(f32)).astype(f32) * LENGTH).astype(f32)).astype(f32)
    limit = ((((w1 + w2).astype(f32) + SKIN).astype(f32) * f32(1.0002)).astype(f32) + SPHERE_EPS).astype(f32)
    return dot(d, d) <= (limit * limit).astype(f32)


def test_sphere_pretest_passes_every_exact_pair():
    rng = np.random.default_rng(5)
    n = 400_000
    r1 = rng.choice([3.5e-6, 9.5e-6], size=n)
    r2 = rng.choice([3.5e-6, 9.5e-6], size=n)
    u1 = unit(rng.normal(size=(n, 3)))
    u2 = unit(rng.normal(size=(n, 3)))
    near = rng.random(n) < 0.4
    tilt = unit(np.cross(u1, rng.normal(size=(n, 3))))
    angle = rng.uniform(0.005, 0.05, size=n)[:, None]
    u2 = np.where(near[:, None], unit(u1 * np.cos(angle) + tilt * np.sin(angle)), u2)
    d1, d2 = u1 * (4.0 * r1)[:, None], u2 * (4.0 * r2)[:, None]
    p1 = rng.uniform(0.0, float(LENGTH), size=(n, 3))
    x1 = p1 + d1 * rng.random(n)[:, None]
    interaction = (r1 + r2 + float(SKIN)) * 1.0001
    sep = unit(rng.normal(size=(n, 3))) * (interaction * rng.uniform(0.9, 1.05, size=n))[:, None]
    p2 = x1 + sep - d2 * rng.random(n)[:, None]
    # The bound's tight case: end to end, nearly collinear, the gap at the
    # interaction distance, so the midpoints are h1 + h2 + gap apart.
    chain = rng.random(n) < 0.3
    bend = rng.uniform(0.0, 0.01, size=n)[:, None]
    v2 = unit(u1 * np.cos(bend) + tilt * np.sin(bend)) * (4.0 * r2)[:, None]
    gap = (interaction * rng.uniform(0.9999, 1.0, size=n))[:, None]
    p2 = np.where(chain[:, None], p1 + d1 + u1 * gap, p2)
    d2 = np.where(chain[:, None], v2, d2)
    wrap1 = rng.integers(-2, 3, size=(n, 3)) * float(LENGTH)
    wrap2 = rng.integers(-2, 3, size=(n, 3)) * float(LENGTH)
    p1, q1 = p1 + wrap1, p1 + d1 + wrap1
    p2, q2 = p2 + wrap2, p2 + d2 + wrap2
    p1, q1, r1, p2, q2, r2 = as_f32(p1, q1, r1, p2, q2, r2)
    exact = exact_build_test(p1, q1, r1, p2, q2, r2)
    sphere = sphere_test(p1, q1, r1, p2, q2, r2)
    assert not np.any(exact & ~sphere)
    assert exact.sum() > 10_000 and (~exact).sum() > 10_000
