"""Needling (crates/tangle_generate/src/recipe.rs:233-300, :1086-1180,
:1688-1812): the reference's known answers for the footprint centre and the
two selection rules (recipe_tests.rs:182-330), and a needled recipe on the
oracle and on CUDA (bit-identical)."""

import numpy as np
import pytest

from tangle_b200.assembly import Cell, FiberAssembly, PackedAssembly
from tangle_b200.generate import ply_collections, ply_stack_specimen
from tangle_b200.needling import (CircularFootprint, NeedlingConfig, RandomFiberFraction, random_footprint_center,
                                  selected_needling_vertices)
from tangle_b200.recipe import Recipe, RecipeError
from tangle_b200.settings import RelaxationSettings


def test_random_footprint_center_is_pinned_deterministic_and_inside():
    """recipe_tests.rs:312-330."""
    center = random_footprint_center(20_260_940, 2, [0.0, 0.0], [1.0e-3, 1.0e-3])
    assert np.float32(center[0]) == np.float32(0.000_797_881_1)
    assert np.float32(center[1]) == np.float32(0.000_692_911_7)
    for layer in (0, 1, 7, 0xFFFFFFFF):
        c = random_footprint_center(11, layer, [-1.0, 2.0], [0.5, 0.25])
        assert c == random_footprint_center(11, layer, [-1.0, 2.0], [0.5, 0.25])
        assert -1.0 <= c[0] < -0.5 and 2.0 <= c[1] < 2.25
    assert random_footprint_center(11, 0, [0.0, 0.0], [1.0, 1.0]) != random_footprint_center(11, 1, [0.0, 0.0],
                                                                                              [1.0, 1.0])


def test_random_selection_is_reproducible_internal_and_layer_scoped():
    """recipe_tests.rs:182-261."""
    assembly = FiberAssembly(Cell([1.0] * 3, ""))
    for index, layer in enumerate((0, 1, 1)):
        assembly.add_fiber([[0.2, 0.2, 0.2], [0.3, 0.2, 0.2], [0.4, 0.2, 0.2], [0.5, 0.2, 0.2]],
                           [[0.0, 0.0, 0.0], [0.1, 0.0, 0.0], [0.2, 0.0, 0.0], [0.3, 0.0, 0.0]], radius=0.01)
        assembly.set_fiber_formation_layer(index, layer)
        assembly.set_fiber_formation_step(index, layer)
    packed = PackedAssembly.from_assembly(assembly)
    config = NeedlingConfig(1, RandomFiberFraction(1.0, seed=42), 0.1, 1.0, 0.1, 0.25)
    active = np.ones(3, dtype=bool)
    first = selected_needling_vertices(assembly, packed, packed.positions, active, 1, 2, config)
    second = selected_needling_vertices(assembly, packed, packed.positions, active, 1, 2, config)
    assert first == second and len(first) == 2
    for vertex in first:
        fiber = vertex // 4
        assert assembly.fibers[fiber].formation_layer == 1
        assert 4 * fiber < vertex < 4 * fiber + 3


def test_circular_footprint_selects_one_internal_vertex_per_fiber_inside():
    """recipe_tests.rs:263-310: only the thick layer-1 fiber through the
    circle qualifies; its vertex nearest the centre is vertex 6."""
    assembly = FiberAssembly(Cell([1.0] * 3, ""))
    for index, (layer, y, radius) in enumerate(((1, 0.5, 0.01), (1, 0.5, 0.02), (0, 0.5, 0.02), (1, 0.8, 0.02))):
        placed = [[0.3, y, 0.5], [0.4, y, 0.5], [0.5, y, 0.5], [0.6, y, 0.5]]
        assembly.add_fiber(placed, placed, radius=radius)
        assembly.set_fiber_formation_layer(index, layer)
        assembly.set_fiber_formation_step(index, layer)
    packed = PackedAssembly.from_assembly(assembly)
    config = NeedlingConfig(1, CircularFootprint([0.5, 0.5], diameter=0.1), 0.1, 1.0, 0.1, 0.25,
                            min_fiber_diameter=0.03)
    selected = selected_needling_vertices(assembly, packed, packed.positions, np.ones(4, dtype=bool), 1, 2, config)
    assert selected == [6]


D = 7.0e-6
THICKNESS = 0.05e-3


def needled_recipe():
    plies = ply_collections(ply_stack_specimen(plies=2, side=0.25e-3, thickness=THICKNESS, fiber_length=0.2e-3,
                                               segment_over_d=2.0, seed=21))
    recipe = Recipe(plies[0].cell)
    recipe.insert(plies[0], name="ply 0")
    recipe.relax_for(16)
    recipe.insert(plies[1], name="ply 1")
    with recipe.needle_layer(1, footprint=RandomFiberFraction(0.5, seed=3), depth=0.3 * THICKNESS, stiffness=0.5,
                             max_translation=0.2 * D):
        recipe.relax_for(24)
    with recipe.needle_layer(1, footprint=CircularFootprint.random(diameter=0.1e-3, seed=5), depth=0.2 * THICKNESS,
                             stiffness=0.5, max_translation=0.2 * D):
        recipe.relax_for(16)
    return recipe


def settings():
    return RelaxationSettings(penetration_tolerance=1.0e-2 * D, max_step=0.2 * D, iterations_per_batch=16)


def oracle_factory(packed, cell_list, max_step):
    from oracle import OracleWorld

    return OracleWorld(packed, cell_list, max_step)


def test_needled_recipe_on_the_oracle():
    recipe = needled_recipe()
    assert recipe.operations()[3].startswith("needle layer 1 through a random 0.5")
    assert recipe.operations()[5] == "release needles"
    result = recipe.run(settings(), world_factory=oracle_factory)
    needles = [e for e in result.events if e.startswith("needle layer 1")]
    assert len(needles) == 2
    assert all(not e.endswith("(0 vertices)") for e in needles), needles
    assert result.iterations == 56


def test_needling_a_layer_not_yet_inserted_stops_the_recipe():
    plies = ply_collections(ply_stack_specimen(plies=2, side=0.25e-3, thickness=THICKNESS, fiber_length=0.2e-3,
                                               segment_over_d=2.0, seed=21))
    recipe = Recipe(plies[0].cell)
    recipe.insert(plies[0])
    recipe.needle_layer(1, footprint=RandomFiberFraction(1.0), depth=1.0e-6)
    with pytest.raises(RecipeError, match="has not been inserted yet"):
        recipe.run(settings(), world_factory=oracle_factory)
    with pytest.raises(ValueError):
        recipe.needle_layer(1, footprint=RandomFiberFraction(1.0), depth=-1.0)
    with pytest.raises(ValueError):
        RandomFiberFraction(0.0)
    with pytest.raises(TypeError):
        recipe.needle_layer(1, footprint="everywhere", depth=1.0e-6)


@pytest.mark.gpu
def test_needled_recipe_on_cuda_matches_the_oracle(cuda_lib):
    oracle_result = needled_recipe().run(settings(), world_factory=oracle_factory)
    cuda_result = needled_recipe().run(settings())
    assert cuda_result.events == oracle_result.events
    for a, b in zip(cuda_result.assembly.fibers, oracle_result.assembly.fibers):
        np.testing.assert_array_equal(a.placed.astype(np.float32).view(np.uint32),
                                      b.placed.astype(np.float32).view(np.uint32))
