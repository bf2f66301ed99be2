"""The contact pass's own filters never drop a pair that produces a hit.

Two filters in tangle_b200/csrc/contact.cuh sit in front of the
reference's closest-point solve and must not change any result:

* `lines_may_touch` drops a pair whose axis lines are farther apart than
  (r1 + r2) x 1.001 + eps; such a pair's solve gives no penetration.
* `within_contact_skin` keeps, at a position snapshot, every pair that can
  overlap before some vertex moves 0.4995 of the contact skin; the listed
  passes only look at kept pairs.

This restates the solve (contact.rs:663-750), the axis distance and both
filters in f32, operation for operation (numpy rounds every f32 operation
and contracts nothing, as the kernels are compiled), and checks both claims
on random pairs near touching at the mid-size specimen's scale: unwrapped
coordinates up to a box length outside the cell, diameters 7 and 19 um,
segments 2 d long, axes from crossed to within 0.005 rad of parallel. The
GPU parity tests check the kernels themselves bit for bit.
"""

import numpy as np

f32 = np.float32
BOX = f32(2.0e-3)
LINE_EPS = f32(4.0e-6) * BOX  # the kernels' line margin: 4e-6 of the largest box edge
R_MAX = f32(9.5e-6)
CONTACT_SKIN = f32(0.1) * (f32(2.0) * R_MAX)  # 0.1 of the neighbor skin (2 r_max)


def dot(u, v):
    return ((u[:, 0] * v[:, 0] + u[:, 1] * v[:, 1]).astype(f32) + u[:, 2] * v[:, 2]).astype(f32)


def clamp01(x):
    return np.clip(x, f32(0.0), f32(1.0)).astype(f32)


def closest(p1, d1, p2, d2, refine_parallel):
    """(s, t) of contact_solve (refine_parallel) or axis_distance."""
    r = (p1 - p2).astype(f32)
    a, e, f = dot(d1, d1), dot(d2, d2), dot(d2, r)
    c, b = dot(d1, r), dot(d1, d2)
    den = (a * e - b * b).astype(f32)
    parallel = np.abs(den) <= (f32(1.0e-6) * a * e).astype(f32)
    with np.errstate(divide="ignore", invalid="ignore"):
        s = np.where(parallel, f32(0.0), clamp01(((b * f - c * e).astype(f32) / den).astype(f32))).astype(f32)
    projected = ((b * s + f).astype(f32) / e).astype(f32)
    low, high = projected < 0.0, projected > 1.0
    s = np.where(low, clamp01((-c / a).astype(f32)), np.where(high, clamp01(((b - c) / a).astype(f32)), s)).astype(f32)
    t = np.where(low, f32(0.0), np.where(high, f32(1.0), projected)).astype(f32)
    if refine_parallel:
        end_projected = ((b + f) / e).astype(f32)
        elow, ehigh = end_projected < 0.0, end_projected > 1.0
        end_s = np.where(elow, clamp01((-c / a).astype(f32)),
                         np.where(ehigh, clamp01(((b - c) / a).astype(f32)), f32(1.0))).astype(f32)
        end_t = np.where(elow, f32(0.0), np.where(ehigh, f32(1.0), end_projected)).astype(f32)
        g = (r + d1 * s[:, None] - d2 * t[:, None]).astype(f32)
        h = (r + d1 * end_s[:, None] - d2 * end_t[:, None]).astype(f32)
        take = parallel & (dot(h, h) < dot(g, g))
        s, t = np.where(take, end_s, s), np.where(take, end_t, t)
    return s, t


def distance(p1, d1, p2, d2, refine_parallel):
    s, t = closest(p1, d1, p2, d2, refine_parallel)
    delta = ((p2 + d2 * t[:, None]).astype(f32) - (p1 + d1 * s[:, None]).astype(f32)).astype(f32)
    return np.sqrt(dot(delta, delta)).astype(f32)


def hits(p1, d1, r1, p2, d2, r2):
    penetration = ((r1 + r2).astype(f32) - distance(p1, d1, p2, d2, True)).astype(f32)
    return penetration > 0.0


def lines_may_touch(p1, d1, r1, p2, d2, r2):
    n = np.stack([(d1[:, 1] * d2[:, 2] - d1[:, 2] * d2[:, 1]), (d1[:, 2] * d2[:, 0] - d1[:, 0] * d2[:, 2]),
                  (d1[:, 0] * d2[:, 1] - d1[:, 1] * d2[:, 0])], 1).astype(f32)
    nn, aa, ee = dot(n, n), dot(d1, d1), dot(d2, d2)
    no_bound = ~(nn > (f32(1.0e-4) * aa * ee).astype(f32))
    rn = dot((p2 - p1).astype(f32), n)
    threshold = ((r1 + r2).astype(f32) * f32(1.001) + LINE_EPS).astype(f32)
    return no_bound | ((rn * rn).astype(f32) <= (threshold * threshold * nn).astype(f32))


def within_contact_skin(p1, d1, r1, p2, d2, r2):
    h1 = (f32(0.5) * np.sqrt(dot(d1, d1))).astype(f32)
    h2 = (f32(0.5) * np.sqrt(dot(d2, d2))).astype(f32)
    threshold = (((r1 + r2).astype(f32) + CONTACT_SKIN).astype(f32) * f32(1.01) +
                 (f32(2.0e-3) * (h1 + h2).astype(f32)).astype(f32) + LINE_EPS).astype(f32)
    return distance(p1, d1, p2, d2, False) <= threshold


def unit(v):
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def pairs_near_touching(rng, n, gap_low, gap_high):
    """Segments whose chosen points are (r1 + r2) x U(gap_low, gap_high) apart."""
    r1 = rng.choice([3.5e-6, 9.5e-6], size=n)
    r2 = rng.choice([3.5e-6, 9.5e-6], size=n)
    u1 = unit(rng.normal(size=(n, 3)))
    u2 = unit(rng.normal(size=(n, 3)))
    near = rng.random(n) < 0.4  # axes 0.005-0.05 rad from parallel
    tilt = unit(np.cross(u1, rng.normal(size=(n, 3))))
    angle = rng.uniform(0.005, 0.05, size=n)[:, None]
    u2 = np.where(near[:, None], unit(u1 * np.cos(angle) + tilt * np.sin(angle)), u2)
    d1 = u1 * (4.0 * r1)[:, None]
    d2 = u2 * (4.0 * r2)[:, None]
    p1 = rng.uniform(-BOX, 2.0 * BOX, size=(n, 3))
    x1 = p1 + d1 * rng.random(n)[:, None]
    sep = unit(rng.normal(size=(n, 3))) * ((r1 + r2) * rng.uniform(gap_low, gap_high, size=n))[:, None]
    p2 = x1 + sep - d2 * rng.random(n)[:, None]
    return p1, d1, r1, p2, d2, r2


def as_f32(*arrays):
    return [np.asarray(x, dtype=np.float32) for x in arrays]


def test_lines_bound_drops_no_hit():
    rng = np.random.default_rng(7)
    p1, d1, r1, p2, d2, r2 = pairs_near_touching(rng, 400_000, 0.9, 1.15)
    q2 = (p2 + d2).astype(np.float32)  # segments travel as end points: d2 = q2 - p2 in f32
    p1, d1, r1, p2, r2 = as_f32(p1, d1, r1, p2, r2)
    d2 = (q2 - p2).astype(f32)
    hit = hits(p1, d1, r1, p2, d2, r2)
    keep = lines_may_touch(p1, d1, r1, p2, d2, r2)
    assert not np.any(hit & ~keep)
    assert hit.sum() > 10_000 and (~keep).sum() > 10_000  # both sides are exercised


def test_contact_lists_keep_every_pair_that_can_touch():
    rng = np.random.default_rng(11)
    n = 400_000
    # Pairs overlapping a little now, traced back to a snapshot from which
    # each end point has moved up to 0.4995 of the contact skin, half of them
    # straight apart (the snapshot as far as the trigger allows).
    p1, d1, r1, p2, d2, r2 = pairs_near_touching(rng, n, 0.97, 1.0)
    q1, q2 = p1 + d1, p2 + d2
    reach = 0.4995 * float(CONTACT_SKIN)
    apart = unit((p2 + 0.5 * d2) - (p1 + 0.5 * d1))
    straight = rng.random(n) < 0.5

    def moved(sign):  # each end point on its own, up to the trigger distance
        m = unit(rng.normal(size=(n, 3))) * (reach * rng.random(n) ** 0.2)[:, None]
        return np.where(straight[:, None], sign * apart * reach, m)

    now = as_f32(p1, q1, p2, q2)
    snap = as_f32(p1 + moved(-1.0), q1 + moved(-1.0), p2 + moved(1.0), q2 + moved(1.0))
    r1, r2 = as_f32(r1, r2)

    def segments(p, q, pp, qq):
        return p, (q - p).astype(f32), pp, (qq - pp).astype(f32)

    a1, e1, a2, e2 = segments(*now)
    hit = hits(a1, e1, r1, a2, e2, r2)
    b1, g1, b2, g2 = segments(*snap)
    keep = within_contact_skin(b1, g1, r1, b2, g2, r2)
    assert not np.any(hit & ~keep)
    assert hit.sum() > 10_000
