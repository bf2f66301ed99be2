"""Formation recipes (crates/tangle_python/src/recipe.rs:240-560 recording,
crates/tangle_generate/src/recipe.rs:859-1600 execution): plies inserted as
formation steps of one resident world, placed above each other with held
layer targets, settled, released, and the walls fitted to the stack.

The recipe runs on the oracle here (`world_factory`); the GPU test runs the
same recipe on the CUDA world and requires the same events, iteration count
and bit-identical centerlines.
"""

import numpy as np
import pytest

from tangle_b200.generate import layer_centers, ply_collections, ply_stack_specimen
from tangle_b200.recipe import Recipe, RecipeError
from tangle_b200.settings import RelaxationSettings

D = 7.0e-6
THICKNESS = 0.05e-3


def stack():
    return ply_stack_specimen(plies=3, side=0.25e-3, thickness=THICKNESS, fiber_length=0.2e-3, segment_over_d=2.0,
                              seed=11)


def settings():
    return RelaxationSettings(penetration_tolerance=1.0e-2 * D, max_step=0.2 * D, iterations_per_batch=16,
                              max_iterations=4000)


def layered_recipe():
    plies = ply_collections(stack())
    recipe = Recipe(plies[0].cell)
    assert recipe.stack_axis == 2
    recipe.insert(plies[0], name="ply 0")
    recipe.relax_for(8)
    for k in (1, 2):
        recipe.insert(plies[k], name=f"ply {k}")
        with recipe.place_layer_above(k, gap=0.6 * THICKNESS, stiffness=0.5, max_translation=0.2 * D):
            recipe.settle_targets(tolerance=0.5 * D, max_iterations=400)
    recipe.set_min_bend_radius("fiber_7um", 6.0 * D)
    recipe.fit_cell_to_active_fibers(padding=0.25 * D)
    recipe.relax_for(8)
    return recipe


def oracle_factory(packed, cell_list, max_step):
    from oracle import OracleWorld

    return OracleWorld(packed, cell_list, max_step)


def test_recipe_records_the_reference_operations():
    recipe = layered_recipe()
    ops = recipe.operations()
    assert ops[0] == "insert 'ply 0' (%d fibers) as formation step 0" % len(ply_collections(stack())[0].fibers)
    assert ops[3] == "place layer 1 above layer 0"
    assert ops[5] == "release layer placement"
    assert ops[-2].startswith("fit cell to active fibers")
    with pytest.raises(ValueError):
        recipe.place_layer_above(0, gap=1.0)
    with pytest.raises(ValueError):
        recipe.scale_layer_spacing(-1.0)
    with pytest.raises(ValueError):
        recipe.settle_targets(tolerance=-1.0, max_iterations=10)
    with pytest.raises(ValueError):
        recipe.fit_cell_to_active_fibers(axes=[True, False, False])  # x is periodic
    with pytest.raises(ValueError):
        recipe.set_min_bend_radius("", 1.0)


def test_ply_by_ply_recipe_on_the_oracle():
    recipe = layered_recipe()
    result = recipe.run(settings(), world_factory=oracle_factory)
    assert result.events == recipe.operations()
    assert result.fiber_count == len(stack().fibers)
    # The walls moved onto the stack, and every vertex lies inside them.
    lengths = result.assembly.cell.lengths
    assert lengths[2] < 3 * THICKNESS
    z = np.concatenate([f.placed[:, 2] for f in result.assembly.fibers])
    lower = result.assembly.cell.origin[2]
    assert z.min() >= lower and z.max() <= lower + lengths[2]
    # The plies stay stacked in order.
    centers = layer_centers(result.assembly, 2)
    assert centers[0] < centers[1] < centers[2]


def test_unknown_material_stops_the_recipe():
    plies = ply_collections(stack())
    recipe = Recipe(plies[0].cell)
    recipe.insert(plies[0])
    recipe.set_min_bend_radius("kevlar", 1.0e-4)
    with pytest.raises(RecipeError, match="unknown material"):
        recipe.run(settings(), world_factory=oracle_factory)


@pytest.mark.gpu
def test_ply_by_ply_recipe_on_cuda_matches_the_oracle(cuda_lib):
    oracle_result = layered_recipe().run(settings(), world_factory=oracle_factory)
    cuda_result = layered_recipe().run(settings())
    assert cuda_result.events == oracle_result.events
    assert cuda_result.iterations == oracle_result.iterations
    assert cuda_result.assembly.cell.lengths == oracle_result.assembly.cell.lengths
    for a, b in zip(cuda_result.assembly.fibers, oracle_result.assembly.fibers):
        np.testing.assert_array_equal(a.placed.astype(np.float32).view(np.uint32),
                                      b.placed.astype(np.float32).view(np.uint32))
