"""The launch-shape autotuner (tgl_autotune, tangle_b200.autotune).

* Every launch shape it chooses among gives the oracle's positions bit for
  bit (the shapes move time, never results).
* A search leaves the world's state as it found it: the positions that
  follow are those of an untuned world, bit for bit, for a single world and
  for an arena.
* The chosen shape comes from the candidate sets, is cached per GPU and
  workload shape, and a second world of the same shape takes it from the
  cache without searching.
"""

import numpy as np
import pytest

from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import batched_specimens, mid_size_specimen
from tangle_b200.settings import RelaxationConfig, RelaxationSettings

pytestmark = pytest.mark.gpu


def small_world_inputs():
    assembly = mid_size_specimen(scale=0.2, seed=3)
    d = assembly.smallest_diameter()
    cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * d, neighbor_capacity=256,
                             max_list_bytes=1 << 30).to_config(d)
    fixed = RelaxationConfig(**{**cfg.__dict__, "force_full_iterations": True})
    return PackedAssembly.from_assembly(assembly), fixed


@pytest.mark.parametrize("params", [
    {"lanes_per_fiber": 4, "contact_blocks_per_sm": 1, "build_chunk": 1024, "contact_skin_fraction": 0.25,
     "update_warps_per_block": 1},
    {"lanes_per_fiber": 32, "contact_blocks_per_sm": 2, "build_chunk": 4096, "contact_skin_fraction": 0.05,
     "update_warps_per_block": 2},
    {"lanes_per_fiber": 2, "contact_blocks_per_sm": 3, "build_chunk": 512, "contact_skin_fraction": 0.0,
     "update_warps_per_block": 4},
], ids=["lanes4", "lanes32", "lanes2_lists_off"])
def test_every_launch_shape_gives_the_oracle_positions(params, cuda_lib):
    from oracle import OracleWorld
    from tangle_b200.device import DeviceWorld

    packed, fixed = small_world_inputs()
    dev = DeviceWorld(packed, fixed.cell_list, fixed.max_step)
    dev.set_launch_params(params)
    got = dev.launch_params()
    keys = ("lanes_per_fiber", "contact_blocks_per_sm", "build_chunk", "update_warps_per_block")
    assert {k: got[k] for k in keys} == {k: params[k] for k in keys}
    orc = OracleWorld(packed, fixed.cell_list, fixed.max_step)
    for batch in (9, 23):
        assert dev.run_batch(fixed, batch).total_iterations == orc.run_batch(fixed, batch).total_iterations
    np.testing.assert_array_equal(dev.download_positions().view(np.uint32), orc.download_positions().view(np.uint32))
    dev.close()
    orc.close()


def test_launch_params_are_validated(cuda_lib):
    from tangle_b200.device import DeviceWorld

    packed, fixed = small_world_inputs()
    dev = DeviceWorld(packed, fixed.cell_list, fixed.max_step)
    good = dev.launch_params()
    for bad in ({"lanes_per_fiber": 16}, {"contact_blocks_per_sm": 4}, {"build_chunk": 8192},
                {"contact_skin_fraction": 1.5}, {"update_warps_per_block": 3}):
        with pytest.raises(ValueError):
            dev.set_launch_params({**good, **bad})
    assert dev.launch_params() == good
    dev.close()


def test_search_leaves_the_world_state_unchanged(cuda_lib, tmp_path):
    from tangle_b200 import autotune as at
    from tangle_b200.device import DeviceWorld

    packed, fixed = small_world_inputs()
    tuned = DeviceWorld(packed, fixed.cell_list, fixed.max_step)
    plain = DeviceWorld(packed, fixed.cell_list, fixed.max_step)
    for world in (tuned, plain):
        world.run_batch(fixed, 37)
    cache = tmp_path / "autotune.json"
    result = at.autotune(tuned, fixed, trial_iterations=8, path=str(cache))
    assert not result["cached"] and result["report"]["trials"] >= 8
    p = result["params"]
    assert p["lanes_per_fiber"] in (2, 4, 8, 32) and p["contact_blocks_per_sm"] in (1, 2, 3)
    assert p["build_chunk"] in (1024, 1536, 2048, 3072, 4096) and p["update_warps_per_block"] in (1, 2, 4)
    assert any(abs(p["contact_skin_fraction"] - v) < 1.0e-6 for v in (0.05, 0.1, 0.15, 0.25))
    assert result["report"]["best_ms"] <= result["report"]["default_ms"]
    a, b = tuned.run_batch(fixed, 41), plain.run_batch(fixed, 41)
    assert (a.total_iterations, a.converged) == (b.total_iterations, b.converged)
    np.testing.assert_array_equal(tuned.download_positions().view(np.uint32),
                                  plain.download_positions().view(np.uint32))
    # A second world of the same shape takes the cached choice.
    again = DeviceWorld(packed, fixed.cell_list, fixed.max_step)
    second = at.autotune(again, fixed, trial_iterations=8, path=str(cache))
    assert second["cached"] and second["params"] == p
    assert again.launch_params()["lanes_per_fiber"] == p["lanes_per_fiber"]
    for world in (tuned, plain, again):
        world.close()


def test_search_on_an_arena_leaves_its_state_unchanged(cuda_lib):
    from tangle_b200.device import DeviceWorld

    assemblies = batched_specimens(count=6, seed=2, max_fibers=300)
    packs = [PackedAssembly.from_assembly(a) for a in assemblies]
    d = min(a.smallest_diameter() for a in assemblies)
    cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * d, neighbor_capacity=256,
                             max_list_bytes=1 << 30).to_config(d)
    fixed = RelaxationConfig(**{**cfg.__dict__, "force_full_iterations": True})
    tuned = DeviceWorld.arena(packs, fixed.cell_list, fixed.max_step)
    plain = DeviceWorld.arena(packs, fixed.cell_list, fixed.max_step)
    for world in (tuned, plain):
        world.run_batch(fixed, 19)
    params, report = tuned.autotune_trials(fixed, 8)
    assert report["trials"] >= 6  # the arena's contact lists are searched too
    assert any(abs(params["contact_skin_fraction"] - v) < 1.0e-6 for v in (0.05, 0.1, 0.15, 0.25))
    tuned.run_batch(fixed, 31)
    plain.run_batch(fixed, 31)
    np.testing.assert_array_equal(tuned.download_positions().view(np.uint32),
                                  plain.download_positions().view(np.uint32))
    tuned.close()
    plain.close()
