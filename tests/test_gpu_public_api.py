"""The reference's public-API relaxation tests, restated on the CUDA path.

Every run goes through `Recipe(...).insert(...).run(settings)` with the
default backend, "cuda" (the library's C ABI), as a user of the Python
surface calls it.

* crates/tangle_python/python/tests/test_api.py:498-542:
  `test_micrometer_fibers_relax_with_default_lengths`,
  `test_segments_shorter_than_the_diameter_converge`,
  `test_insert_a_population_and_run`;
* examples/biased_fiber_box/tests/population_regression.rs:15-62: seeded
  biased populations in a walled unit box (160 fibers of 8 segments, lengths
  0.4-0.58, radii 0.012-0.017, rest waviness up to 0.014, bend radius at
  least 0.08) relax with the flexible model within 6,000 iterations to
  max penetration <= 1e-4 and curvature ratio <= 1 + 1e-5, and keep their
  orientation bias: the length-weighted orientation tensor moves by less
  than 0.05 (Frobenius), the isotropic case keeps every diagonal entry in
  [0.15, 0.55) and the aligned case keeps Axx > 0.9. The planar-layered case
  of that regression runs the layered formation before its final solve and
  is not restated here.

The reference's populations come from its own generator
(crates/tangle_generate/src/population.rs), restated in
tangle_b200.generate; the random draws are this library's SplitMix64
stream, so the specimens are statistically, not bitwise, the reference's.
"""

import math

import numpy as np
import pytest

from tangle_b200 import Recipe, RelaxationSettings
from tangle_b200.assembly import Cell, Material
from tangle_b200.generate import (FiberPopulation, biased_fiber_population, generate_fiber_population,
                                  orientation_tensor)
from tangle_b200.settings import RelaxationConfig

um = 1.0e-6


def run(recipe, factory, settings=None):
    """Recipe.run on the CUDA world (factory None) or on `factory`'s world."""
    return recipe.run(settings) if factory is None else recipe.run(settings, world_factory=factory)


def check_micrometer_fibers_relax_with_default_lengths(factory=None):
    # Unset lengths follow the fiber diameter, so 10 um fibers need no
    # hand-tuned settings.
    fiber = Material("fiber", diameter=10 * um)
    population = FiberPopulation(material=fiber, count=20)
    assert population.length is None
    assert RelaxationSettings().penetration_tolerance is None
    cell = Cell([400 * um] * 3, periodic="xyz")
    collection = generate_fiber_population(cell, population)
    for line in collection.centerlines():
        length = sum(math.dist(a, b) for a, b in zip(line, line[1:]))
        assert length < 25 * 10 * um
    recipe = Recipe(cell)
    recipe.insert(collection)
    recipe.relax_until_converged()
    result = run(recipe, factory)
    assert result.converged
    assert result.max_penetration <= 0.01 * 10 * um


def check_segments_shorter_than_the_diameter_converge(factory=None):
    fiber = Material("fiber", diameter=10 * um)
    population = FiberPopulation(material=fiber, count=5, length=60 * um, segments_per_fiber=16,
                                 curvature_amplitude=0.0)
    cell = Cell([300 * um] * 3, periodic="xyz")
    recipe = Recipe(cell)
    recipe.insert(generate_fiber_population(cell, population))
    recipe.relax_until_converged()
    result = run(recipe, factory)
    assert result.converged


def check_insert_a_population_and_run(factory=None):
    # The shortest path: insert a population, run, and it is relaxed.
    cell = Cell([300 * um] * 3, periodic="xyz")
    fiber = Material("fiber", diameter=10 * um)
    recipe = Recipe(cell)
    recipe.insert(FiberPopulation(material=fiber, count=15))
    assert len(recipe.operations()) == 1
    result = run(recipe, factory)
    assert result.fiber_count == 15
    assert result.converged
    assert "converged=True" in repr(result)
    assert repr(fiber) == 'Material(name="fiber", diameter=1e-05)'
    with pytest.raises(TypeError):
        recipe.insert([[0, 0, 0], [1, 0, 0]])


CASES = {
    "isotropic_3d": ("isotropic",),
    "aligned_x": ("aligned", [1.0, 0.0, 0.0], 15.0 * math.pi / 180.0),
}


def check_relaxed_population_retains_its_material_bias(case, factory=None):
    cell = Cell([1.0, 1.0, 1.0], periodic="")
    assembly = biased_fiber_population(cell, count=160, segments_per_fiber=8, seed=20_260_918,
                                       length=(0.4, 0.58), radius=(0.012, 0.017), curvature_amplitude=(0.0, 0.014),
                                       orientation=CASES[case], min_bend_radius=0.08)
    initial = orientation_tensor(assembly.centerlines())
    recipe = Recipe(cell)
    recipe.insert(assembly)
    recipe.relax_until_converged(max_iterations=6000)
    # RelaxationConfig::flexible().with_iteration_limits(6_000, 128), in the
    # box's own units: the reference's defaults, given as absolute lengths.
    config = RelaxationConfig()
    settings = RelaxationSettings(penetration_tolerance=config.penetration_tolerance, max_step=config.max_step,
                                  max_iterations=6000, iterations_per_batch=128)
    result = run(recipe, factory, settings)
    assert result.converged, f"{case} did not converge"
    assert result.max_penetration <= 1.0e-4
    assert result.max_curvature_ratio <= 1.0 + 1.0e-5
    final = orientation_tensor(result.centerlines())
    for tensor in (initial, final):
        assert abs(np.trace(tensor) - 1.0) < 1.0e-10
    assert float(np.sqrt(((final - initial) ** 2).sum())) < 0.05, f"{case} changed orientation bias"
    if case == "isotropic_3d":
        assert all(0.15 <= final[a, a] < 0.55 for a in range(3))
    else:
        assert final[0, 0] > 0.9


@pytest.mark.gpu
def test_micrometer_fibers_relax_with_default_lengths(cuda_lib):
    check_micrometer_fibers_relax_with_default_lengths()


@pytest.mark.gpu
def test_segments_shorter_than_the_diameter_converge(cuda_lib):
    check_segments_shorter_than_the_diameter_converge()


@pytest.mark.gpu
def test_insert_a_population_and_run(cuda_lib):
    check_insert_a_population_and_run()


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_relaxed_populations_retain_their_material_bias(case, cuda_lib):
    check_relaxed_population_retains_its_material_bias(case)
