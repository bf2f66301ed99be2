"""Geometries of the reference's relaxation tests, restated.

Each builder cites the fixture it restates in
crates/tangle_relax/src/device/world_tests.rs (reference project).
"""

import math

import numpy as np

from tangle_b200.assembly import Cell, FiberAssembly, PackedAssembly


def crossed_assembly():
    """world_tests.rs:8-21: two crossing capsules, radius 0.1, walled 4^3 box."""
    a = FiberAssembly(Cell([4.0] * 3, ""))
    a.add_fiber([[1.0, 2.0, 2.0], [3.0, 2.0, 2.0]], radius=0.1)
    a.add_fiber([[2.0, 1.0, 2.0], [2.0, 3.0, 2.0]], radius=0.1)
    return a


def single_fiber(points, radius=0.1, min_bend_radius=None, intrinsic=None, box=4.0):
    """world_tests.rs:266-280."""
    a = FiberAssembly(Cell([box] * 3, ""))
    a.add_fiber(points, intrinsic, radius=radius, min_bend_radius=min_bend_radius)
    return a


def short_segments_fiber():
    """world_tests.rs:283-289: twenty 0.05-long segments of a 0.2-diameter fiber."""
    return single_fiber([[1.0 + 0.05 * i, 2.0, 2.0] for i in range(21)])


def hairpin():
    """world_tests.rs:303-312: two 1.5-long legs 0.1 apart."""
    points = [[1.0 + 0.1 * i, 2.0, 2.0] for i in range(16)]
    points += [[1.0 + 0.1 * i, 2.1, 2.0] for i in reversed(range(16))]
    return single_fiber(points)


def dense_cell():
    """world_tests.rs:430-442: three coincident short segments in one
    high-index cell of a long thin box (more than one 256-cell scan block)."""
    a = FiberAssembly(Cell([40.0, 0.2, 0.2], ""))
    for _ in range(3):
        a.add_fiber([[39.0, 0.1, 0.1], [39.01, 0.1, 0.1]], radius=0.02)
    return a


def bent_three_vertex(box=2.0):
    """world_tests.rs:461-483: a 3-vertex fiber bent past its 0.25 bend radius."""
    a = FiberAssembly(Cell([box] * 3, ""))
    a.add_fiber([[0.8, 1.0, 1.0], [1.0, 1.15, 1.0], [1.2, 1.0, 1.0]],
                [[-0.15, 0.0, 0.0], [0.0, 0.0, 0.0], [0.15, 0.0, 0.0]], radius=0.01, min_bend_radius=0.25)
    return a


def min_image_pair():
    """world_tests.rs:934-947: fibers at x=0.05 and x=3.95 of a box periodic in x."""
    a = FiberAssembly(Cell([4.0] * 3, "x"))
    for x in (0.05, 3.95):
        a.add_fiber([[x, 1.5, 2.0], [x, 2.5, 2.0]], radius=0.1)
    return a


def si_scale_crossing():
    """world_tests.rs:972-987: 20 um fibers crossing in a 2 mm walled box."""
    a = FiberAssembly(Cell([0.002] * 3, ""))
    a.add_fiber([[0.0006, 0.001, 0.001], [0.0014, 0.001, 0.001]], radius=10.0e-6)
    a.add_fiber([[0.001, 0.0006, 0.001], [0.001, 0.0014, 0.001]], radius=10.0e-6)
    return a


def unwrapped_images():
    """world_tests.rs:999-1013: the second fiber lies two box images away."""
    a = FiberAssembly(Cell([0.0025, 0.0025, 0.002], "xy"))
    a.add_fiber([[0.0005, 0.0006, 0.001], [0.0005, 0.0014, 0.001]], radius=10.0e-6)
    a.add_fiber([[0.0051, 0.001, 0.001], [0.0059, 0.001, 0.001]], radius=10.0e-6)
    return a


def self_image_loop():
    """world_tests.rs:1029-1045: one fiber touching its own periodic image."""
    a = FiberAssembly(Cell([4.0] * 3, "x"))
    a.add_fiber([[0.05, 1.0, 2.0], [0.05, 1.5, 2.0], [2.0, 1.5, 2.0], [3.95, 1.5, 2.0], [3.95, 1.0, 2.0]],
                radius=0.1)
    return a


def pinned_zigzag():
    """world_tests.rs:1126-1157: pinned 81-vertex zig-zag, every interior
    vertex past its 0.3 bend radius."""
    intrinsic = [[0.02 * i, 0.0, 0.0] for i in range(81)]
    placed = [[0.2 + 0.02 * i, 1.0 + (0.0 if i % 2 == 0 else 0.01), 1.0] for i in range(81)]
    a = FiberAssembly(Cell([2.0] * 3, ""))
    a.add_fiber(placed, intrinsic, radius=0.005, min_bend_radius=0.3)
    return a


def dense_crossed_mat():
    """world_tests.rs:1262-1287: 24 fibers x 8 segments, periodic in x and y."""
    a = FiberAssembly(Cell([2.4, 2.4, 1.0], "xy"))
    for index in range(12):
        offset = 0.05 + 0.18 * index
        wobble = 0.03 * (index % 3)
        along_x = [[0.2 + 0.25 * p, offset, 0.45 + wobble] for p in range(9)]
        along_y = [[offset + 0.07, 0.2 + 0.25 * p, 0.55 - wobble] for p in range(9)]
        a.add_fiber(along_x, radius=0.1)
        a.add_fiber(along_y, radius=0.1)
    return a


def host_segment_axis_distance(p1, q1, p2, q2):
    """world_tests.rs:1365-1397: f64 axis distance on the host."""
    d1 = q1 - p1
    d2 = q2 - p2
    r = p1 - p2
    a, e, f, c, b = d1 @ d1, d2 @ d2, d2 @ r, d1 @ r, d1 @ d2
    den = a * e - b * b
    s = min(max((b * f - c * e) / den, 0.0), 1.0) if den > 1.0e-12 * a * e else 0.0
    t = (b * s + f) / e
    if t < 0.0:
        t = 0.0
        s = min(max(-c / a, 0.0), 1.0)
    elif t > 1.0:
        t = 1.0
        s = min(max((b - c) / a, 0.0), 1.0)
    delta = p2 + d2 * t - p1 - d1 * s
    return math.sqrt(delta @ delta)
