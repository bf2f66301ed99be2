"""capture_segment_contacts (contact.rs:9-230; world.rs:2195-2335).

The reference's known answers (world_tests.rs:933-1064: one contact across
a periodic face at gap -0.1; an SI-scale interior crossing at -20 um; a
pair several box lengths apart reduced to its minimum image, -20 um), then
a brute-force f64 check on a random specimen: the same pair set (pairs
within 1e-4 d of the threshold excepted), gaps within 1e-4 d, crossing
angles within 1e-3 rad, and closest-point parameters within 1e-3 where
the axes are not nearly parallel.
"""

import numpy as np
import pytest

import fixtures as fx
from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import mid_size_specimen
from tangle_b200.settings import CellListConfig, RelaxationConfig

pytestmark = pytest.mark.gpu


def world_of(assembly, max_step):
    from tangle_b200.device import DeviceWorld

    return DeviceWorld(PackedAssembly.from_assembly(assembly), CellListConfig(), max_step)


def test_periodic_broad_phase_captures_minimum_image_contact(cuda_lib):
    w = world_of(fx.min_image_pair(), 0.1)
    capture = w.capture_contacts(0.0, 16)
    assert not capture.overflow
    assert len(capture.candidates) == 1
    assert abs(capture.candidates[0].surface_gap + 0.1) < 1.0e-5
    # world_tests.rs:957-967: the relaxation after a capture still converges.
    config = RelaxationConfig(penetration_tolerance=1.0e-5, correction_fraction=0.8, max_step=0.05,
                              max_iterations=40, iterations_per_batch=40)
    status = w.run_batch(config, 40)
    assert status.converged and status.max_penetration <= config.penetration_tolerance


def test_si_scale_interior_crossing(cuda_lib):
    capture = world_of(fx.si_scale_crossing(), 1.0e-6).capture_contacts(0.0, 16)
    assert not capture.overflow and len(capture.candidates) == 1
    c = capture.candidates[0]
    assert abs(c.surface_gap + 20.0e-6) < 0.01e-6
    assert abs(c.crossing_angle - np.pi / 2) < 1e-3


def test_periodic_contact_reduces_multiple_unwrapped_box_images(cuda_lib):
    capture = world_of(fx.unwrapped_images(), 1.0e-6).capture_contacts(0.0, 16)
    assert not capture.overflow and len(capture.candidates) == 1
    assert abs(capture.candidates[0].surface_gap + 20.0e-6) < 0.01e-6


def test_capture_overflow_is_reported(cuda_lib):
    assembly = mid_size_specimen(scale=0.12, seed=9)
    capture = world_of(assembly, 1.0e-7).capture_contacts(0.5 * assembly.smallest_diameter(), 4)
    assert capture.overflow and len(capture.candidates) == 4


def brute_force(packed, max_gap):
    x = packed.positions.reshape(-1, 3).astype(np.float64)
    sv = packed.segment_vertices.reshape(-1, 2)
    fib = packed.segment_fibers
    r = packed.segment_radii.astype(np.float64)
    box = (packed.cell_upper - packed.cell_lower).astype(np.float64)
    per = packed.cell_periodic.astype(bool)
    p, q = x[sv[:, 0]], x[sv[:, 1]]
    mid = 0.5 * (p + q)
    S = len(fib)
    out = {}
    for a in range(S):
        b = np.arange(a + 1, S)
        b = b[fib[b] != fib[a]]
        sep = mid[b] - mid[a]
        sep -= np.where(per, np.round(sep / box) * box, 0.0)
        reach = 0.5 * np.linalg.norm(q[a] - p[a]) + 0.5 * np.linalg.norm(q[b] - p[b], axis=1) + r[a] + r[b] + max_gap
        b = b[np.linalg.norm(sep, axis=1) <= reach * 1.01]
        for o in b:
            p2, q2 = p[o].copy(), q[o].copy()
            d = 0.5 * (p2 + q2 - p[a] - q[a])
            shift = np.where(per, np.round(d / box) * box, 0.0)
            p2 -= shift
            q2 -= shift
            d1, d2, rr = q[a] - p[a], q2 - p2, p[a] - p2
            A, E, F, C, B = d1 @ d1, d2 @ d2, d2 @ rr, d1 @ rr, d1 @ d2
            den = A * E - B * B
            s = min(max((B * F - C * E) / den, 0.0), 1.0) if abs(den) > 1e-6 * A * E else 0.0
            t = (B * s + F) / E
            if t < 0.0:
                t, s = 0.0, min(max(-C / A, 0.0), 1.0)
            elif t > 1.0:
                t, s = 1.0, min(max((B - C) / A, 0.0), 1.0)
            gap = np.linalg.norm(rr + d1 * s - d2 * t) - r[a] - r[o]
            angle = np.arccos(min(abs(B) / np.sqrt(A * E), 1.0))
            out[(a, int(o))] = (s, t, gap, angle)
    return out


def test_capture_matches_an_f64_brute_force(cuda_lib):
    assembly = mid_size_specimen(scale=0.12, seed=9)
    packed = PackedAssembly.from_assembly(assembly)
    d = assembly.smallest_diameter()
    max_gap = 0.2 * d
    w = world_of(assembly, 0.05 * d)
    capture = w.capture_contacts(max_gap, 1 << 20)
    assert not capture.overflow
    got = {(c.first_segment, c.second_segment): c for c in capture.candidates}
    keys = [(c.first_segment, c.second_segment, c.first_coordinate, c.second_coordinate)
            for c in capture.candidates]
    assert keys == sorted(keys)
    ref = brute_force(packed, max_gap)
    near = {k for k, v in ref.items() if abs(v[2] - max_gap) < 1e-4 * d}
    expected = {k for k, v in ref.items() if v[2] <= max_gap}
    assert set(got) - near == expected - near
    assert len(expected) > 50
    for k in set(got) & expected:
        s, t, gap, angle = ref[k]
        c = got[k]
        assert abs(c.surface_gap - gap) < 1e-4 * d, k
        assert abs(c.crossing_angle - angle) < 1e-3, k
        if abs(angle) > 1e-2:  # parameters are ill-defined for nearly parallel axes
            assert abs(c.first_coordinate - s) < 1e-3 and abs(c.second_coordinate - t) < 1e-3, k
