"""The reference's relaxation known-answer tests, on the oracle and on CUDA.

Each test restates one test of crates/tangle_relax/src/device/world_tests.rs
(cited per test) with the same geometry, settings and thresholds. The
"oracle" parameter pins the CPU restatement against the reference's own
expectations; the "cuda" parameter (marked gpu) holds the B200 path to the
same expectations.
"""

import math

import numpy as np
import pytest

import fixtures as fx
from tangle_b200.assembly import PackedAssembly
from tangle_b200.settings import CellListConfig, RelaxationConfig

BACKENDS = [pytest.param("oracle", id="oracle"), pytest.param("cuda", id="cuda", marks=pytest.mark.gpu)]


def make_world(kind, assembly, max_step, cell_list=None, pin_ends=False, pin_all=False):
    packed = PackedAssembly.from_assembly(assembly, pin_ends)
    if pin_all:
        packed.vertex_pinned[:] = 1
    cell_list = cell_list or CellListConfig()
    if kind == "oracle":
        from oracle import OracleWorld

        return OracleWorld(packed, cell_list, max_step)
    from tangle_b200.build import build
    from tangle_b200.device import DeviceWorld

    build()
    return DeviceWorld(packed, cell_list, max_step)


@pytest.mark.parametrize("kind", BACKENDS)
def test_flexible_crossed_fibers_relax(kind):
    """world_tests.rs:23-45: converged within 20 iterations."""
    w = make_world(kind, fx.crossed_assembly(), 0.2)
    cfg = RelaxationConfig(penetration_tolerance=1.0e-5, correction_fraction=1.0, max_step=0.2)
    st = w.run_batch(cfg, 20)
    assert st.converged, st
    assert st.total_iterations > 0
    assert st.max_penetration <= cfg.penetration_tolerance


@pytest.mark.parametrize("kind", BACKENDS)
def test_segments_shorter_than_the_diameter_do_not_touch_their_own_fiber(kind):
    """world_tests.rs:282-300."""
    w = make_world(kind, fx.short_segments_fiber(), 0.2)
    cfg = RelaxationConfig(penetration_tolerance=1.0e-5, max_step=0.02)
    st = w.run_batch(cfg, 50)
    assert st.converged, st
    assert st.max_penetration <= cfg.penetration_tolerance


@pytest.mark.parametrize("kind", BACKENDS)
def test_a_fiber_folded_onto_itself_is_pushed_apart(kind):
    """world_tests.rs:302-332: real self-contact is resolved."""
    w = make_world(kind, fx.hairpin(), 0.2)
    cfg = RelaxationConfig(penetration_tolerance=1.0e-4, max_step=0.02)
    st = w.run_batch(cfg, 4000)
    assert st.max_penetration < 0.01, st
    p = w.download_positions().reshape(-1, 3)
    gap = float(np.sqrt(((p[0] - p[-1]).astype(np.float32) ** 2).sum()))
    assert gap >= 0.2 - 1.0e-3


@pytest.mark.parametrize("kind", BACKENDS)
def test_fully_pinned_overlap_is_not_accepted(kind):
    """world_tests.rs:334-355: the gate refuses an overlap nothing can move."""
    w = make_world(kind, fx.crossed_assembly(), 0.2, pin_ends=True)
    cfg = RelaxationConfig(penetration_tolerance=1.0e-5, correction_fraction=1.0, max_step=0.2)
    st = w.run_batch(cfg, 5)
    assert not st.converged
    assert st.max_penetration > cfg.penetration_tolerance


@pytest.mark.parametrize("kind", BACKENDS)
def test_compact_cell_list_accepts_dense_cells(kind):
    """world_tests.rs:429-458: more than one scan block, one crowded cell."""
    w = make_world(kind, fx.dense_cell(), 0.01)
    assert w.cell_count > 256
    cfg = RelaxationConfig(max_step=0.01)
    st = w.run_batch(cfg, 5)
    assert not st.cell_list_overflow
    assert math.isfinite(st.max_penetration)


@pytest.mark.parametrize("kind", BACKENDS)
def test_curvature_limit_moves_a_free_middle_between_pinned_ends(kind):
    """world_tests.rs:460-509: ends bit-identical, middle pulled down."""
    w = make_world(kind, fx.bent_three_vertex(), 0.02, pin_ends=True)
    cfg = RelaxationConfig(penetration_tolerance=1.0e-5, correction_fraction=0.8, stretch_stiffness=0.0,
                           bend_stiffness=0.0, curvature_limit_stiffness=1.0, curvature_ratio_tolerance=1.0e-5,
                           constraint_iterations=1, max_step=0.02)
    st = w.run_batch(cfg, 40)
    assert st.converged, st
    assert st.max_curvature_ratio <= 1.0 + 1.0e-5
    p = w.download_positions()
    assert list(p[0:3]) == [np.float32(0.8), np.float32(1.0), np.float32(1.0)]
    assert list(p[6:9]) == [np.float32(1.2), np.float32(1.0), np.float32(1.0)]
    assert p[4] < np.float32(1.15)


@pytest.mark.parametrize("kind", BACKENDS)
def test_fully_pinned_bend_violation_is_not_accepted(kind):
    """world_tests.rs:511-554."""
    w = make_world(kind, fx.bent_three_vertex(), 0.02, pin_all=True)
    cfg = RelaxationConfig(stretch_stiffness=0.0, bend_stiffness=0.0, curvature_limit_stiffness=1.0,
                           curvature_ratio_tolerance=1.0e-5, constraint_iterations=1)
    st = w.run_batch(cfg, 5)
    assert not st.converged
    assert st.max_curvature_ratio > 1.0 + cfg.curvature_ratio_tolerance


@pytest.mark.parametrize("kind", BACKENDS)
def test_periodic_broad_phase_captures_minimum_image_contact(kind):
    """world_tests.rs:933-969: overlap 0.1 across the periodic x face."""
    w = make_world(kind, fx.min_image_pair(), 0.1)
    cfg = RelaxationConfig(penetration_tolerance=1.0e-5, correction_fraction=0.8, max_step=0.05)
    _, pen = w.debug_corrections(cfg)
    assert abs(float(pen.max()) - 0.1) < 1.0e-5
    st = w.run_batch(cfg, 40)
    assert st.converged, st
    assert st.max_penetration <= cfg.penetration_tolerance


@pytest.mark.parametrize("kind", BACKENDS)
def test_si_scale_interior_crossing_is_not_misclassified_as_parallel(kind):
    """world_tests.rs:971-996: surface gap -20 um within 0.01 um."""
    w = make_world(kind, fx.si_scale_crossing(), 1.0e-6)
    cfg = RelaxationConfig(max_step=1.0e-6)
    _, pen = w.debug_corrections(cfg)
    assert abs(float(pen.max()) - 20.0e-6) < 0.01e-6


@pytest.mark.parametrize("kind", BACKENDS)
def test_periodic_contact_reduces_multiple_unwrapped_box_images(kind):
    """world_tests.rs:998-1026."""
    w = make_world(kind, fx.unwrapped_images(), 1.0e-6)
    cfg = RelaxationConfig(max_step=1.0e-6)
    _, pen = w.debug_corrections(cfg)
    assert abs(float(pen.max()) - 20.0e-6) < 0.01e-6


@pytest.mark.parametrize("kind", BACKENDS)
def test_periodic_broad_phase_resolves_nonadjacent_self_image_contact(kind):
    """world_tests.rs:1028-1064."""
    w = make_world(kind, fx.self_image_loop(), 0.1)
    cfg = RelaxationConfig(penetration_tolerance=1.0e-4, correction_fraction=0.8, max_step=0.05)
    first = w.run_batch(cfg, 1)
    assert first.max_penetration > 0.05, first
    st = w.run_batch(cfg, 999)
    assert st.max_penetration < 0.005, st


@pytest.mark.parametrize("kind", BACKENDS)
def test_curvature_cleanup_straightens_a_long_zigzag_in_few_iterations(kind):
    """world_tests.rs:1159-1188: Gauss-Seidel converges within 30."""
    w = make_world(kind, fx.pinned_zigzag(), 0.02, pin_ends=True)
    cfg = RelaxationConfig(penetration_tolerance=1.0e-5, stretch_stiffness=0.0, bend_stiffness=0.0,
                           curvature_limit_stiffness=1.0, curvature_ratio_tolerance=1.0e-5,
                           constraint_iterations=1, curvature_cleanup_sweeps=1, max_step=0.02)
    st = w.run_batch(cfg, 30)
    assert st.converged, st
    assert st.max_curvature_ratio <= 1.0 + 1.0e-5
    p = w.download_positions()
    assert list(p[0:3]) == [np.float32(0.2), np.float32(1.0), np.float32(1.0)]
    assert list(p[240:243]) == [np.float32(1.8), np.float32(1.0), np.float32(1.0)]


def relax_dense_mat(kind, cell_list):
    """world_tests.rs:1289-1307."""
    w = make_world(kind, fx.dense_crossed_mat(), 0.01, cell_list)
    cfg = RelaxationConfig(penetration_tolerance=0.0, force_full_iterations=True, max_step=0.01)
    st = w.run_batch(cfg, 40)
    assert math.isfinite(st.max_penetration)
    return w.download_positions(), w.neighbor_list_rebuilds()


@pytest.mark.parametrize("kind", BACKENDS)
def test_neighbor_lists_match_rebuilding_every_iteration(kind):
    """world_tests.rs:1309-1340: skin lists and the overflow scan agree with
    rebuilding every iteration to 1e-4, and the skin saves rebuilds."""
    reference, reference_rebuilds = relax_dense_mat(kind, CellListConfig(neighbor_skin_scale=0.0))
    listed, listed_rebuilds = relax_dense_mat(kind, CellListConfig())
    overflowed, _ = relax_dense_mat(kind, CellListConfig(neighbor_capacity=1))
    assert np.abs(listed - reference).max() < 1.0e-4
    assert np.abs(overflowed - reference).max() < 1.0e-4
    assert listed_rebuilds < reference_rebuilds


@pytest.mark.parametrize("kind", BACKENDS)
def test_neighbor_lists_hold_every_pair_within_the_skin(kind):
    """world_tests.rs:1399-1485: lists against an f64 host closest-point oracle
    with a 0.1 % band around the cutoff."""
    assembly = fx.dense_crossed_mat()
    packed = PackedAssembly.from_assembly(assembly)
    w = make_world(kind, assembly, 0.01)
    w.run_batch(RelaxationConfig(max_step=0.01), 1)
    _, lists = w.debug_neighbor_lists()
    skin = float(w.neighbor_skin)
    pos = packed.positions.astype(np.float64).reshape(-1, 3)
    sv = packed.segment_vertices.reshape(-1, 2)
    lengths = np.array([2.4, 2.4, 1.0])
    periodic = [True, True, False]
    segments = packed.segment_count
    checked = 0
    for first in range(segments):
        listed = lists[first]
        assert listed is not None, f"segment {first} overflowed"
        assert len(set(listed.tolist())) == len(listed), f"segment {first} lists a neighbor twice"
        a, b = sv[first]
        p1, q1 = pos[a], pos[b]
        listed_set = set(listed.tolist())
        for second in range(segments):
            c, d = sv[second]
            adjacent = packed.segment_fibers[first] == packed.segment_fibers[second] and len({a, b} & {c, d}) > 0
            if second == first or adjacent:
                assert second not in listed_set
                continue
            p2, q2 = pos[c].copy(), pos[d].copy()
            for axis in range(3):
                if periodic[axis]:
                    shift = round(0.5 * (p2[axis] + q2[axis] - p1[axis] - q1[axis]) / lengths[axis]) * lengths[axis]
                    p2[axis] -= shift
                    q2[axis] -= shift
            interaction = float(packed.segment_radii[first]) + float(packed.segment_radii[second]) + skin
            distance = fx.host_segment_axis_distance(p1, q1, p2, q2)
            if distance < 0.999 * interaction:
                assert second in listed_set, f"{first}-{second} at {distance} missing"
                checked += 1
            elif distance > 1.001 * interaction:
                assert second not in listed_set, f"{first}-{second} at {distance} listed"
    assert checked > segments


@pytest.mark.parametrize("kind", BACKENDS)
def test_relaxation_is_bitwise_repeatable(kind):
    """world_tests.rs:1487-1510, with lists and with the overflow scan."""
    for cell_list in (CellListConfig(), CellListConfig(neighbor_capacity=1)):
        first, first_rebuilds = relax_dense_mat(kind, cell_list)
        second, second_rebuilds = relax_dense_mat(kind, cell_list)
        assert first_rebuilds == second_rebuilds
        assert first.view(np.uint32).tolist() == second.view(np.uint32).tolist()
