"""FP64 restatement of the contact distances -- test infrastructure.

Only tests and the bench's checking legs use this module, as the checker of
the f32 contact pass: it is never on the product path.

The reference checks its neighbor lists against a host closest-point oracle
in f64 (crates/tangle_relax/src/device/world_tests.rs:1364-1485,
`host_segment_axis_distance` and `neighbor_lists_hold_every_pair_within_the_skin`).
This module restates that oracle, vectorised with numpy:

* `segment_axis_distance` -- world_tests.rs:1365-1397: the distance
  between two segment axes (clamped closest-point parameters, parallel axes
  when a e - b^2 <= 1e-12 a e);
* `minimum_image` -- world_tests.rs:1449-1457 (and neighbor.rs:301-318):
  the second segment shifted by the rounded midpoint separation on every
  periodic axis;
* `penetration` -- crates/tangle_contact/src/device/contact.rs:741:
  r1 + r2 - distance; a segment's maximum penetration is the largest
  positive one over its contacts (0 when it has none), contact.rs:749-753.

`spot_check` compares a contact pass's per-segment maximum penetration
(f32) with the f64 value over the segment's listed neighbors, and checks in
f64 that every pair within the neighbor skin of a sampled segment is listed
(the 0.1 % band of world_tests.rs:1470-1479 around the cutoff).
"""

from __future__ import annotations

import numpy as np


def segment_axis_distance(p1, q1, p2, q2):
    """world_tests.rs:1365-1397 in f64, over arrays of shape (n, 3)."""
    p1, q1, p2, q2 = (np.asarray(x, dtype=np.float64) for x in (p1, q1, p2, q2))
    d1 = q1 - p1
    d2 = q2 - p2
    r = p1 - p2
    a = np.einsum("ij,ij->i", d1, d1)
    e = np.einsum("ij,ij->i", d2, d2)
    f = np.einsum("ij,ij->i", d2, r)
    c = np.einsum("ij,ij->i", d1, r)
    b = np.einsum("ij,ij->i", d1, d2)
    denominator = a * e - b * b
    with np.errstate(divide="ignore", invalid="ignore"):
        s = np.where(denominator > 1.0e-12 * a * e, np.clip((b * f - c * e) / denominator, 0.0, 1.0), 0.0)
        t = (b * s + f) / e
        low = t < 0.0
        high = t > 1.0
        s = np.where(low, np.clip(-c / a, 0.0, 1.0), s)
        s = np.where(high, np.clip((b - c) / a, 0.0, 1.0), s)
        t = np.where(low, 0.0, np.where(high, 1.0, t))
    delta = p2 + d2 * t[:, None] - p1 - d1 * s[:, None]
    return np.sqrt(np.einsum("ij,ij->i", delta, delta))


def minimum_image(p1, q1, p2, q2, lengths, periodic):
    """world_tests.rs:1449-1457: shift the second segment by whole box
    lengths so its midpoint is nearest the first's, per periodic axis."""
    p2 = np.array(p2, dtype=np.float64, copy=True)
    q2 = np.array(q2, dtype=np.float64, copy=True)
    for axis in range(3):
        if periodic[axis]:
            length = float(lengths[axis])
            shift = np.round(0.5 * (p2[:, axis] + q2[:, axis] - p1[:, axis] - q1[:, axis]) / length) * length
            p2[:, axis] -= shift
            q2[:, axis] -= shift
    return p2, q2


def _segment_points(positions, segment_vertices, segments):
    x = np.asarray(positions, dtype=np.float32).reshape(-1, 3).astype(np.float64)
    sv = np.asarray(segment_vertices, dtype=np.int64).reshape(-1, 2)
    return x[sv[segments, 0]], x[sv[segments, 1]]


def pair_distances(packed, positions, first, second):
    """f64 axis distances of segment pairs (first[i], second[i]) under the
    minimum image of the packed cell."""
    lengths = np.asarray(packed.cell_upper, dtype=np.float64) - np.asarray(packed.cell_lower, dtype=np.float64)
    periodic = [bool(x) for x in packed.cell_periodic]
    p1, q1 = _segment_points(positions, packed.segment_vertices, first)
    p2, q2 = _segment_points(positions, packed.segment_vertices, second)
    p2, q2 = minimum_image(p1, q1, p2, q2, lengths, periodic)
    return segment_axis_distance(p1, q1, p2, q2)


def listed_pairs(counts, lists, block, segments):
    """(first, second) arrays of the listed pairs of `segments` from a
    block-strided list array; segments whose list overflowed are skipped."""
    segments = np.asarray(segments, dtype=np.int64)
    n = np.asarray(counts, dtype=np.int64)[segments]
    keep = n <= block
    segments, n = segments[keep], n[keep]
    first = np.repeat(segments, n)
    starts = np.repeat(segments * block, n)
    within = np.arange(first.size, dtype=np.int64) - np.repeat(np.cumsum(n) - n, n)
    second = np.asarray(lists, dtype=np.int64)[starts + within]
    return first, second, segments


def max_penetrations(packed, positions, first, second, segments):
    """Per segment of `segments`: the largest positive r1 + r2 - d64 over its
    pairs (0 with none), contact.rs:741-753 in f64."""
    radii = np.asarray(packed.segment_radii, dtype=np.float32).astype(np.float64)
    pen = radii[first] + radii[second] - pair_distances(packed, positions, first, second)
    index = np.searchsorted(segments, first)
    out = np.zeros(segments.size, dtype=np.float64)
    np.maximum.at(out, index, np.where(pen > 0.0, pen, 0.0))
    return out


def f32_bound(positions, lengths):
    """The f32 rounding bound used for penetrations: 16 units in the last
    place of the largest coordinate magnitude (unwrapped coordinates, plus one
    box length for a minimum-image shift). The f32 pass computes the closest
    points' difference from coordinates of that magnitude, a handful of
    roundings each; the distance is stationary in the closest-point
    parameters, so their rounding adds only second-order error."""
    magnitude = float(np.abs(np.asarray(positions, dtype=np.float64)).max()) + float(np.max(lengths))
    return 16.0 * float(np.spacing(np.float32(magnitude)))


def arc_lengths(packed):
    """Rest arc length of every vertex (f64 accumulate, then f32:
    crates/tangle_relax/src/device/packed.rs:561-580)."""
    x = np.asarray(packed.intrinsic_positions, dtype=np.float32).reshape(-1, 3).astype(np.float64)
    arc = np.zeros(packed.vertex_count, dtype=np.float32)
    for start, count in np.asarray(packed.fiber_vertex_spans, dtype=np.int64).reshape(-1, 2):
        if count < 2:
            continue
        steps = np.sqrt(((x[start + 1: start + count] - x[start: start + count - 1]) ** 2).sum(axis=1))
        arc[start + 1: start + count] = np.cumsum(steps).astype(np.float32)
    return arc


def missing_pairs_within_skin(packed, positions, counts, lists, block, segments, skin):
    """Pairs of the sampled `segments` whose f64 axis distance is below
    0.999 (r1 + r2 + skin) but that are not listed (world_tests.rs:1470-1479),
    excluding the pairs the build skips: the segment itself and its
    near-along-fiber neighbors (same fiber, arc gap below r1 + r2,
    neighbor.rs:169-240). Candidates come from a periodic k-d tree over the
    segment midpoints (reach: both half lengths plus both radii plus the
    skin). Returns an array of (first, second) rows."""
    from scipy.spatial import cKDTree

    lower = np.asarray(packed.cell_lower, dtype=np.float64)
    lengths = np.asarray(packed.cell_upper, dtype=np.float64) - lower
    periodic = np.asarray(packed.cell_periodic, dtype=bool)
    S = int(packed.segment_count)
    everything = np.arange(S)
    p, q = _segment_points(positions, packed.segment_vertices, everything)
    mid = 0.5 * (p + q)
    half = 0.5 * np.sqrt(((q - p) ** 2).sum(axis=1))
    radii = np.asarray(packed.segment_radii, dtype=np.float32)
    reach = 2.0 * float(half.max()) + 2.0 * float(radii.max()) + float(skin)
    boxed = mid - lower
    if periodic.all():
        tree = cKDTree(np.mod(boxed, lengths), boxsize=lengths)
        queries = np.mod(boxed[segments], lengths)
    else:
        # A walled axis: plain coordinates, and the periodic axes' images by
        # brute repetition would be needed; every specimen checked here is
        # periodic on all axes or walled on all axes.
        assert not periodic.any(), "mixed periodic and walled axes are not supported here"
        tree = cKDTree(boxed)
        queries = boxed[segments]
    candidates = tree.query_ball_point(queries, r=reach)
    first = np.repeat(np.asarray(segments, dtype=np.int64), [len(c) for c in candidates])
    second = np.concatenate([np.asarray(c, dtype=np.int64) for c in candidates]) if len(candidates) else first
    keep = first != second
    first, second = first[keep], second[keep]
    fibers = np.asarray(packed.segment_fibers, dtype=np.int64)
    arc = arc_lengths(packed)
    sv = np.asarray(packed.segment_vertices, dtype=np.int64).reshape(-1, 2)
    gap = np.maximum(arc[sv[second, 0]] - arc[sv[first, 1]], arc[sv[first, 0]] - arc[sv[second, 1]])
    near_along = (fibers[first] == fibers[second]) & (gap < radii[first] + radii[second])
    first, second = first[~near_along], second[~near_along]
    distance = pair_distances(packed, positions, first, second)
    interaction = radii[first].astype(np.float64) + radii[second].astype(np.float64) + float(skin)
    inside = distance < 0.999 * interaction
    first, second = first[inside], second[inside]
    lf, ls, _ = listed_pairs(counts, lists, block, np.unique(first))
    listed = set(zip(lf.tolist(), ls.tolist()))
    overflowed = np.asarray(counts, dtype=np.int64)[first] > block
    missing = [(a, b) for a, b, o in zip(first.tolist(), second.tolist(), overflowed.tolist())
               if not o and (a, b) not in listed]
    return np.asarray(missing, dtype=np.int64).reshape(-1, 2), int(first.size)


def spot_check(packed, positions, counts, lists, block, penetration32, segments, skin):
    """The f64 checks on the sampled `segments`. Returns a dict: the largest
    |pen32 - pen64| over the sample (m), the bound it is held to, the number
    of sampled segments in contact, the pairs within the skin checked and the
    ones missing from the lists."""
    segments = np.unique(np.asarray(segments, dtype=np.int64))
    first, second, kept = listed_pairs(counts, lists, block, segments)
    pen64 = max_penetrations(packed, positions, first, second, kept)
    pen32 = np.asarray(penetration32, dtype=np.float32)[kept].astype(np.float64)
    lengths = np.asarray(packed.cell_upper, dtype=np.float64) - np.asarray(packed.cell_lower, dtype=np.float64)
    missing, within = missing_pairs_within_skin(packed, positions, counts, lists, block, segments, skin)
    error = np.abs(pen32 - pen64)
    worst = int(np.argmax(error)) if error.size else 0
    return {
        "segments": int(kept.size),
        "pairs": int(first.size),
        "in_contact": int((pen64 > 0.0).sum()),
        "max_abs_error": float(error.max()) if error.size else 0.0,
        "worst_segment": int(kept[worst]) if error.size else -1,
        "bound": f32_bound(positions, lengths),
        "pairs_within_skin": within,
        "missing": missing,
    }
