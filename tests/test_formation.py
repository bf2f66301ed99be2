"""Formation hooks: staged activation, layer and vertex targets, cell
compaction and its metrics, per-fiber curvature limits.

* The reference's known answers (crates/tangle_relax/src/device/
  world_tests.rs, cited per test), on the oracle and on CUDA.
* Parity: a layered, walled stack deposited ply by ply -- activation of
  each ply, persistent and single-layer targets, vertex targets under both
  motion models, wall and affine compaction, new curvature limits -- with
  the CUDA path and the oracle bit-identical after every batch (positions,
  statuses, rebuild counts, wall reactions, target errors, cell bounds).
  The compaction metrics sum f32 terms in f64 on the device and serially in
  f32 in the oracle (as the reference does): they agree within 2e-4
  relative.
* A checkpoint taken with targets installed, a compacted cell and frozen
  plies restores into a world that continues bit-identically.
"""

import numpy as np
import pytest

from tangle_b200.assembly import Cell, FiberAssembly, PackedAssembly
from tangle_b200.formation import CompactionEnergyModel, CompactionKinematics
from tangle_b200.generate import layer_centers, ply_stack_specimen
from tangle_b200.settings import CellListConfig, RelaxationConfig

from test_known_answers import BACKENDS

import fixtures as fx


def world_of(kind, packed, max_step, cell_list=None):
    cell_list = cell_list or CellListConfig()
    if kind == "oracle":
        from oracle import OracleWorld

        return OracleWorld(packed, cell_list, max_step)
    from tangle_b200.build import build
    from tangle_b200.device import DeviceWorld

    build()
    return DeviceWorld(packed, cell_list, max_step)


def two_layer_assembly(z_first, z_second, steps=False):
    """world_tests.rs:557-580: two straight fibers in a walled unit box,
    layers 0 and 1 at heights z_first and z_second."""
    assembly = FiberAssembly(Cell([1.0] * 3, ""))
    for index, (layer, z) in enumerate(((0, z_first), (1, z_second))):
        assembly.add_fiber([[0.4, 0.5, z], [0.6, 0.5, z]], [[0.0, 0.0, 0.0], [0.2, 0.0, 0.0]], radius=0.01)
        assembly.set_fiber_formation_layer(index, layer)
        if steps:
            assembly.set_fiber_formation_step(index, layer)
    return assembly


# --------------------------------------------------------------- known answers


@pytest.mark.parametrize("kind", BACKENDS)
def test_formation_steps_activate_prepacked_fibers(kind):
    """world_tests.rs:47-75."""
    assembly = fx.crossed_assembly()
    assembly.set_fiber_formation_step(1, 1)
    w = world_of(kind, PackedAssembly.from_assembly(assembly), 0.2)
    assert w.activate_formation_step(0) == (1, 2)
    first = fx.crossed_assembly()
    w.unpack_positions(w.download_positions(), first)
    assert len(first.fibers) == 1
    assert np.allclose(first.fibers[0].placed, [[1.0, 2.0, 2.0], [3.0, 2.0, 2.0]])
    assert w.activate_formation_step(1) == (2, 4)
    second = fx.crossed_assembly()
    w.unpack_positions(w.download_positions(), second)
    assert len(second.fibers) == 2


@pytest.mark.parametrize("kind", BACKENDS)
def test_layer_target_command_updates_resident_geometry(kind):
    """world_tests.rs:556-587."""
    w = world_of(kind, PackedAssembly.from_assembly(two_layer_assembly(0.2, 0.8)), 0.01)
    w.apply_layer_targets(2, [0.3, 0.7], 1.0, 1.0)
    z = w.download_positions().reshape(-1, 3)[:, 2]
    assert np.all(np.abs(z[:2] - 0.3) < 1.0e-6)
    assert np.all(np.abs(z[2:] - 0.7) < 1.0e-6)


@pytest.mark.parametrize("kind", BACKENDS)
def test_single_layer_target_leaves_the_relaxed_stack_free(kind):
    """world_tests.rs:589-624."""
    w = world_of(kind, PackedAssembly.from_assembly(two_layer_assembly(0.24, 0.8)), 0.01)
    w.apply_single_layer_target(2, [0.2, 0.7], 1, 1.0, 1.0)
    error = w.formation_target_error()
    assert error.vertex is None
    assert error.layer < 1.0e-6
    p = w.download_positions()
    assert abs(p[2] - 0.24) < 1.0e-6 and abs(p[5] - 0.24) < 1.0e-6
    assert abs(p[8] - 0.7) < 1.0e-6 and abs(p[11] - 0.7) < 1.0e-6


@pytest.mark.parametrize("kind", BACKENDS)
def test_layer_targets_do_not_move_inactive_future_layers(kind):
    """world_tests.rs:626-658."""
    w = world_of(kind, PackedAssembly.from_assembly(two_layer_assembly(0.2, 0.8, steps=True)), 0.01)
    w.activate_formation_step(0)
    w.apply_layer_targets(2, [0.3, 0.7], 1.0, 1.0)
    p = w.download_positions()
    assert abs(p[2] - 0.3) < 1.0e-6
    assert abs(p[8] - 0.8) < 1.0e-6


@pytest.mark.parametrize("kind", BACKENDS)
def test_vertex_displacement_target_is_initialized_from_resident_geometry(kind):
    """world_tests.rs:660-696."""
    assembly = FiberAssembly(Cell([1.0] * 3, ""))
    assembly.add_fiber([[0.4, 0.5, 0.5], [0.5, 0.5, 0.5], [0.6, 0.5, 0.5]],
                       [[0.0, 0.0, 0.0], [0.1, 0.0, 0.0], [0.2, 0.0, 0.0]], radius=0.01)
    w = world_of(kind, PackedAssembly.from_assembly(assembly), 0.1)
    w.apply_vertex_displacement_targets(2, [1], -0.1, 1.0, 0.2)
    error = w.formation_target_error()
    assert error.layer is None
    assert abs(error.vertex - 0.1) < 1.0e-6
    w.run_batch(RelaxationConfig(motion_model="rigid_translation", force_full_iterations=True), 1)
    assert abs(w.formation_target_error().vertex) < 1.0e-6
    p = w.download_positions()
    assert abs(p[5] - 0.4) < 1.0e-6 and abs(p[2] - 0.5) < 1.0e-6 and abs(p[8] - 0.5) < 1.0e-6


@pytest.mark.parametrize("kind", BACKENDS)
def test_vertex_displacement_command_advances_independently_of_mechanics(kind):
    """world_tests.rs:698-745."""
    assembly = FiberAssembly(Cell([2.0] * 3, ""))
    assembly.add_fiber([[0.8, 1.0, 1.0], [1.0, 1.0, 1.0], [1.2, 1.0, 1.0]],
                       [[-0.15, 0.0, 0.0], [0.0, 0.0, 0.0], [0.15, 0.0, 0.0]], radius=0.01, min_bend_radius=0.25)
    w = world_of(kind, PackedAssembly.from_assembly(assembly, pin_fiber_ends=True), 0.02)
    w.apply_vertex_displacement_targets(1, [1], -0.05, 1.0, 0.01)
    config = RelaxationConfig(force_full_iterations=True, stretch_stiffness=1.0, bend_stiffness=1.0,
                              curvature_limit_stiffness=1.0, constraint_iterations=4)
    w.run_batch(config, 3)
    target = w.vertex_target_checkpoint()
    assert abs(target.coordinates[0] - 0.95) < 1.0e-6
    assert abs(target.command_coordinates[0] - 0.97) < 1.0e-6
    assert abs(w.download_positions()[4] - 0.97) < 1.0e-6


@pytest.mark.parametrize("kind", BACKENDS)
def test_persistent_layer_targets_are_independent_of_batch_boundaries(kind):
    """world_tests.rs:746-785."""
    assembly = FiberAssembly(Cell([1.0] * 3, ""))
    assembly.add_fiber([[0.4, 0.5, 0.2], [0.6, 0.5, 0.2]], [[0.0, 0.0, 0.0], [0.2, 0.0, 0.0]], radius=0.01)
    assembly.set_fiber_formation_layer(0, 0)
    packed = PackedAssembly.from_assembly(assembly)
    config = RelaxationConfig(force_full_iterations=True)

    def run(batches):
        w = world_of(kind, packed, 0.01)
        w.apply_layer_targets(2, [0.8], 0.2, 1.0)
        for iterations in batches:
            w.run_batch(config, iterations)
        return w.download_positions()

    np.testing.assert_array_equal(run([2, 3]), run([5]))


def one_fiber_box():
    assembly = FiberAssembly(Cell([4.0] * 3, ""))
    assembly.add_fiber([[1.0, 1.0, 1.0], [2.0, 1.0, 1.0]], radius=0.1)
    return PackedAssembly.from_assembly(assembly)


@pytest.mark.parametrize("kind", BACKENDS)
def test_rigid_center_compaction_updates_cell_without_straining_fibers(kind):
    """world_tests.rs:877-904."""
    w = world_of(kind, one_fiber_box(), 0.1)
    w.compact_cell([0.0, 0.0, 0.0], [2.0, 4.0, 4.0], CompactionKinematics.RIGID_FIBER_CENTERS)
    assert w.cell_bounds() == ([0.0, 0.0, 0.0], [2.0, 4.0, 4.0])
    p = w.download_positions()
    assert abs(p[3] - p[0] - 1.0) < 1.0e-6
    assert abs(0.5 * (p[0] + p[3]) - 0.75) < 1.0e-6


@pytest.mark.parametrize("kind", BACKENDS)
def test_affine_compaction_scales_centerline_with_cell(kind):
    """world_tests.rs:906-931."""
    w = world_of(kind, one_fiber_box(), 0.1)
    w.compact_cell([0.0, 0.0, 0.0], [2.0, 4.0, 4.0], CompactionKinematics.AFFINE_VERTICES)
    p = w.download_positions()
    assert abs(p[3] - p[0] - 0.5) < 1.0e-6


@pytest.mark.parametrize("kind", BACKENDS)
def test_curvature_limit_reaches_vertices_packed_after_dormant_fibers(kind):
    """world_tests.rs:1066-1124: a dormant 200-vertex fiber packed first."""
    assembly = FiberAssembly(Cell([2.0] * 3, ""))
    dormant = [[0.1 + 0.004 * i, 0.2, 0.2] for i in range(200)]
    assembly.add_fiber(dormant, radius=0.01)
    assembly.set_fiber_formation_step(0, 1)
    assembly.add_fiber([[0.8, 1.0, 1.0], [1.0, 1.15, 1.0], [1.2, 1.0, 1.0]],
                       [[-0.15, 0.0, 0.0], [0.0, 0.0, 0.0], [0.15, 0.0, 0.0]], radius=0.01, min_bend_radius=0.25)
    w = world_of(kind, PackedAssembly.from_assembly(assembly, pin_fiber_ends=True), 0.02)
    assert w.activate_formation_step(0) == (2, 3)
    config = RelaxationConfig(penetration_tolerance=1.0e-5, correction_fraction=0.8, stretch_stiffness=0.0,
                              bend_stiffness=0.0, curvature_limit_stiffness=1.0, curvature_ratio_tolerance=1.0e-5,
                              constraint_iterations=1, max_step=0.02, max_iterations=40, iterations_per_batch=40)
    status = w.run_batch(config, 40)
    assert status.converged, status
    assert status.max_curvature_ratio <= 1.0 + 1.0e-5


def test_formation_arguments_are_validated():
    """The reference's asserts (world.rs:1750, :1774-1777, :1819-1828,
    :1937-1950) as ValueError, on the oracle (the checks are host-side)."""
    w = world_of("oracle", PackedAssembly.from_assembly(two_layer_assembly(0.2, 0.8)), 0.01)
    with pytest.raises(ValueError):
        w.apply_layer_targets(3, [0.3, 0.7], 1.0, 1.0)
    with pytest.raises(ValueError):
        w.apply_layer_targets(2, [], 1.0, 1.0)
    with pytest.raises(ValueError):
        w.apply_layer_targets(2, [0.3], 1.5, 1.0)
    with pytest.raises(ValueError):
        w.apply_single_layer_target(2, [0.3], 1, 1.0, 1.0)
    with pytest.raises(ValueError):
        w.apply_vertex_displacement_targets(2, [1], 0.0, 1.0, 0.1)
    with pytest.raises(ValueError):
        w.apply_vertex_displacement_targets(2, [99], 0.1, 1.0, 0.1)
    with pytest.raises(ValueError):
        w.compact_cell([0.0, 0.0, 0.0], [1.5, 1.0, 1.0], CompactionKinematics.AFFINE_VERTICES)  # grows
    with pytest.raises(ValueError):
        w.compact_cell([0.0, 0.0, 0.0], [0.01, 1.0, 1.0], CompactionKinematics.AFFINE_VERTICES)  # below 2 radii
    with pytest.raises(ValueError):
        w.compaction_metrics(0.0)
    with pytest.raises(ValueError):
        w.set_fiber_maximum_curvatures([1.0])
    assert w.formation_target_error().layer is None and w.formation_target_error().vertex is None


def test_ply_stack_layout():
    a = ply_stack_specimen(plies=2)
    p = PackedAssembly.from_assembly(a)
    assert a.cell.periodic == [True, True, False]
    assert set(p.fiber_formation_steps.tolist()) == {0, 1}
    assert np.array_equal(p.fiber_formation_steps, p.fiber_formation_layers)
    assert 140_000 < p.segment_count / 2 < 155_000
    assert p.fiber_vertex_spans.reshape(-1, 2)[:, 1].max() <= 256
    centers = layer_centers(a, 2)
    assert len(centers) == 2 and 0.0 < centers[0] < centers[1] < 0.2e-3
    z = np.concatenate([f.placed[:, 2] for f in a.fibers])
    r = np.concatenate([np.full(len(f.placed), f.radius) for f in a.fibers])
    assert np.all(z - r >= -1e-12) and np.all(z + r <= 0.2e-3 + 1e-12)  # every fiber inside the walls


# --------------------------------------------------------------------- parity


def small_stack():
    return ply_stack_specimen(plies=3, side=0.25e-3, thickness=0.05e-3, fiber_length=0.2e-3, segment_over_d=2.0,
                              seed=5)


def compare(orc, dev, label):
    po, pd = orc.download_positions(), dev.download_positions()
    np.testing.assert_array_equal(po.view(np.uint32), pd.view(np.uint32), err_msg=label)
    ro, rd = orc.wall_reactions(), dev.wall_reactions()
    np.testing.assert_array_equal(ro.view(np.uint32), rd.view(np.uint32), err_msg=label + " reactions")
    assert orc.neighbor_list_rebuilds() == dev.neighbor_list_rebuilds(), label
    assert orc.cell_bounds() == dev.cell_bounds(), label
    eo, ed = orc.formation_target_error(), dev.formation_target_error()
    assert (eo.layer, eo.vertex) == (ed.layer, ed.vertex), label


def run_both(orc, dev, config, iterations, label):
    so = orc.run_batch(config, iterations)
    sd = dev.run_batch(config, iterations)
    assert (so.total_iterations, so.batch_iterations) == (sd.total_iterations, sd.batch_iterations), label
    assert np.float32(so.max_penetration) == np.float32(sd.max_penetration), label
    assert np.float32(so.max_curvature_ratio) == np.float32(sd.max_curvature_ratio), label
    compare(orc, dev, label)


def metrics_close(orc, dev, label):
    model = CompactionEnergyModel(2.0, 0.5, 0.25)
    mo, md = orc.compaction_metrics(0.8, model), dev.compaction_metrics(0.8, model)
    got = np.array(list(md.pressure) + [md.contact_energy, md.stretch_energy, md.bending_energy, md.total_energy]
                   + sum(dev.wall_face_pressures(), []))
    ref = np.array(list(mo.pressure) + [mo.contact_energy, mo.stretch_energy, mo.bending_energy, mo.total_energy]
                   + sum(orc.wall_face_pressures(), []))
    np.testing.assert_allclose(got, ref, rtol=2e-4, atol=1e-30, err_msg=label)
    return ref


def deposit_stack(orc, dev, stack):
    """The formation sequence both parity tests drive."""
    d = 7.0e-6
    thickness = 0.05e-3
    flexible = RelaxationConfig(penetration_tolerance=1.0e-3 * d, max_step=0.2 * d, force_full_iterations=True)
    rigid = RelaxationConfig(**{**flexible.__dict__, "motion_model": "rigid_translation"})
    targets = [0.9 * c for c in layer_centers(stack, 2)]
    counts = [w.activate_formation_step(0) for w in (orc, dev)]
    assert counts[0] == counts[1]
    for w in (orc, dev):
        w.apply_layer_targets(2, targets, 0.2, 0.05 * d)
    compare(orc, dev, "ply 0 placed")
    run_both(orc, dev, flexible, 7, "ply 0 relaxed")
    for w in (orc, dev):
        w.activate_formation_step(1)
        w.apply_single_layer_target(2, targets, 1, 0.5, 0.1 * d)
    run_both(orc, dev, flexible, 9, "ply 1 relaxed")
    spans = np.asarray(orc._packed.fiber_vertex_spans).reshape(-1, 2)
    ply2 = [int(f) for f in np.nonzero(np.asarray(orc._packed.fiber_formation_steps) == 2)[0][:4]]
    needles = [int(spans[f, 0] + spans[f, 1] // 2) for f in ply2]
    for w in (orc, dev):
        w.activate_formation_step(2)
        w.apply_vertex_displacement_targets(2, needles, -0.3 * thickness, 0.3, 0.05 * d)
    run_both(orc, dev, rigid, 5, "needled, rigid")
    run_both(orc, dev, flexible, 6, "needled, flexible")
    for w in (orc, dev):
        w.clear_layer_targets()
    run_both(orc, dev, flexible, 4, "layer target released")
    lower, upper = orc.cell_bounds()
    for w in (orc, dev):
        w.compact_cell([lower[0], lower[1], lower[2] + 0.02 * thickness],
                       [upper[0], upper[1], upper[2] - 0.1 * thickness], CompactionKinematics.MOVING_WALLS)
    compare(orc, dev, "wall compaction")
    run_both(orc, dev, flexible, 7, "relaxed after wall compaction")
    return flexible


@pytest.mark.gpu
def test_ply_by_ply_formation_matches_the_oracle_bit_for_bit(cuda_lib):
    stack = small_stack()
    packed = PackedAssembly.from_assembly(stack)
    d = 7.0e-6
    cell_list = CellListConfig()
    orc, dev = world_of("oracle", packed, 0.2 * d, cell_list), world_of("cuda", packed, 0.2 * d, cell_list)
    flexible = deposit_stack(orc, dev, stack)
    metrics_close(orc, dev, "metrics after wall compaction")
    lower, upper = orc.cell_bounds()
    side = upper[0] - lower[0]
    for kinematics in (CompactionKinematics.AFFINE_VERTICES, CompactionKinematics.RIGID_FIBER_CENTERS):
        for w in (orc, dev):
            w.compact_cell(lower, [lower[0] + 0.98 * side, lower[1] + 0.98 * side, upper[2]], kinematics)
        compare(orc, dev, f"compaction {kinematics.name}")
        run_both(orc, dev, flexible, 5, f"relaxed after {kinematics.name}")
        lower, upper = orc.cell_bounds()
        side = upper[0] - lower[0]
    limits = np.full(packed.fiber_count, 1.0 / (4.0 * d), dtype=np.float32)
    for w in (orc, dev):
        w.set_fiber_maximum_curvatures(limits)
        w.clear_vertex_targets()
    run_both(orc, dev, flexible, 6, "new curvature limits")
    metrics_close(orc, dev, "final metrics")
    reactions = dev.wall_reactions().reshape(-1, 3)
    assert np.any(reactions[:, 2] != 0.0)  # the walls pushed back


@pytest.mark.gpu
def test_checkpoint_carries_the_formation_state(cuda_lib, tmp_path):
    from tangle_b200 import checkpoint as ck
    from tangle_b200.device import DeviceWorld

    stack = small_stack()
    packed = PackedAssembly.from_assembly(stack)
    d = 7.0e-6
    orc, dev = world_of("oracle", packed, 0.2 * d), world_of("cuda", packed, 0.2 * d)
    flexible = deposit_stack(orc, dev, stack)
    for w in (orc, dev):  # a held target and a held needle across the save
        w.activate_formation_step(1)
        w.apply_single_layer_target(2, layer_centers(stack, 2), 1, 0.5, 0.1 * d)
    run_both(orc, dev, flexible, 3, "before the save")
    dev.apply_vertex_displacement_targets(2, [3, 40], 0.1 * d, 0.5, 0.02 * d)
    saved = ck.RunCheckpoint("stack", dev.checkpoint(), 0, 0, False)
    path = tmp_path / "stack.ckpt"
    ck.save(path, saved)
    loaded = ck.load(path, "stack")
    restored = DeviceWorld.restore(flexible, loaded.device)
    assert restored.cell_bounds() == dev.cell_bounds()
    assert np.array_equal(restored.fiber_active, dev.fiber_active)
    np.testing.assert_array_equal(restored.wall_reactions(), dev.wall_reactions())
    for w in (dev, restored):
        w.run_batch(flexible, 8)
    np.testing.assert_array_equal(restored.download_positions().view(np.uint32),
                                  dev.download_positions().view(np.uint32))
    e1, e2 = restored.formation_target_error(), dev.formation_target_error()
    assert (e1.layer, e1.vertex) == (e2.layer, e2.vertex)


@pytest.mark.gpu
def test_frozen_fibers_stay_out_of_later_rebuilds(cuda_lib):
    """Freezing deposited plies leaves their Verlet lists behind, unused;
    several rebuilds later, and after the plies thaw again, the relaxation is
    still the oracle's bit for bit and the lists of the segments in the cell
    list are the oracle's."""
    stack = small_stack()
    packed = PackedAssembly.from_assembly(stack)
    d = 7.0e-6
    orc, dev = world_of("oracle", packed, 0.2 * d), world_of("cuda", packed, 0.2 * d)
    flexible = deposit_stack(orc, dev, stack)
    for w in (orc, dev):
        w.activate_formation_step(0)
    for k in range(3):
        run_both(orc, dev, flexible, 3, f"frozen plies, rebuild {k}")
        for w in (orc, dev):
            w.debug_rebuild()
    active = np.asarray(dev.fiber_active, dtype=bool)
    on = active[np.asarray(packed.segment_fibers)]
    oc, ol = orc.debug_neighbor_lists()
    dc, dl = dev.debug_neighbor_lists()
    for s in np.nonzero(on)[0]:
        assert oc[s] == dc[s]
        if ol[s] is not None:
            np.testing.assert_array_equal(ol[s], dl[s])
    for w in (orc, dev):
        w.activate_formation_step(2)
    run_both(orc, dev, flexible, 5, "plies thawed")
