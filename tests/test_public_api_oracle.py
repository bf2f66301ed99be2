"""The reference's public-API relaxation tests (test_api.py:498-542) and its
population regression (population_regression.rs:15-62) on the oracle: the
same checks as test_gpu_public_api.py, run through Recipe.run with the
oracle's world in place of the CUDA world. They pin the oracle to the
reference's own convergence and orientation-bias thresholds."""

import pytest

import test_gpu_public_api as api


def oracle_world(packed, cell_list, max_step):
    from oracle import OracleWorld

    return OracleWorld(packed, cell_list, max_step)


def test_micrometer_fibers_relax_with_default_lengths_on_the_oracle():
    api.check_micrometer_fibers_relax_with_default_lengths(oracle_world)


def test_segments_shorter_than_the_diameter_converge_on_the_oracle():
    api.check_segments_shorter_than_the_diameter_converge(oracle_world)


def test_insert_a_population_and_run_on_the_oracle():
    api.check_insert_a_population_and_run(oracle_world)


@pytest.mark.parametrize("case", sorted(api.CASES))
def test_relaxed_populations_retain_their_material_bias_on_the_oracle(case):
    api.check_relaxed_population_retains_its_material_bias(case, oracle_world)
