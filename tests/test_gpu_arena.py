"""Batched relaxation: an arena of specimens relaxes each of them exactly as
its own world would.

Contract: after the same batches, every specimen's positions in the arena
are bit-identical to the same specimen relaxed alone, its gate stops it at
the same iteration (per-specimen convergence masks), and its neighbor-list
rebuilds are the same.
"""

import numpy as np
import pytest

import fixtures as fx
from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import batched_specimens, cpu_runnable_specimen, mid_size_specimen
from tangle_b200.settings import CellListConfig, RelaxationConfig, RelaxationSettings

pytestmark = pytest.mark.gpu


def mixed_specimens():
    """Different boxes, diameters, periodicity and sizes."""
    return [
        cpu_runnable_specimen(seed=1),
        mid_size_specimen(scale=0.12, seed=2),
        cpu_runnable_specimen(seed=3),
        fx.dense_crossed_mat(),
        mid_size_specimen(scale=0.1, seed=4),
    ]


def config_for(max_step=0.01, tolerance=1.0e-8, force=True):
    return RelaxationConfig(penetration_tolerance=tolerance, max_step=max_step, force_full_iterations=force,
                            cell_list=CellListConfig(neighbor_capacity=256, max_list_bytes=1 << 32))


def test_arena_positions_match_single_worlds_bit_for_bit(cuda_lib):
    from tangle_b200.device import DeviceWorld

    specimens = mixed_specimens()
    packeds = [PackedAssembly.from_assembly(a) for a in specimens]
    cfg = config_for(max_step=RelaxationSettings().to_config(7.0e-6).max_step)
    arena = DeviceWorld.arena(packeds, cfg.cell_list, cfg.max_step)
    singles = [DeviceWorld(p, cfg.cell_list, cfg.max_step) for p in packeds]
    for batch in (7, 13):
        st = arena.run_batch(cfg, batch)
        for w in singles:
            w.run_batch(cfg, batch)
        assert st.batch_iterations == batch
    for i, (got, w) in enumerate(zip(arena.specimen_positions(), singles)):
        np.testing.assert_array_equal(got.view(np.uint32), w.download_positions().view(np.uint32),
                                      err_msg=f"specimen {i}")
    statuses = arena.specimen_statuses(cfg)
    assert [s.total_iterations for s in statuses] == [20] * len(specimens)
    assert arena.neighbor_list_rebuilds() == sum(w.neighbor_list_rebuilds() for w in singles)


@pytest.mark.parametrize("ranked", [None, "1"])
def test_arena_gates_stop_each_specimen_on_its_own(ranked, cuda_lib, monkeypatch):
    """With ranked "1" the update ranks its fibers by their sweep rounds
    before every launch (stopped specimens' fibers rank last, at zero
    rounds): the bits do not change."""
    from tangle_b200.device import DeviceWorld

    if ranked is not None:
        monkeypatch.setenv("TGL_UPDATE_ORDER_PERIOD", "1")
        monkeypatch.setenv("TGL_UPDATE_ORDER_RANKED", ranked)

    specimens = [cpu_runnable_specimen(seed=s) for s in (5, 6, 7)] + [fx.crossed_assembly(), fx.hairpin()]
    packeds = [PackedAssembly.from_assembly(a) for a in specimens]
    # Loose enough that the specimens converge at different iterations.
    cfg = RelaxationConfig(penetration_tolerance=2.0e-7, max_step=1.0e-6,
                           cell_list=CellListConfig(neighbor_capacity=256, max_list_bytes=1 << 32))
    arena = DeviceWorld.arena(packeds, cfg.cell_list, cfg.max_step)
    singles = [DeviceWorld(p, cfg.cell_list, cfg.max_step) for p in packeds]
    budget = 300
    arena.run_batch(cfg, budget)
    per_spec = arena.specimen_statuses(cfg)
    single = [w.run_batch(cfg, budget) for w in singles]
    for i, (a, s) in enumerate(zip(per_spec, single)):
        assert (a.total_iterations, a.converged) == (s.total_iterations, s.converged), i
        assert np.float32(a.max_penetration) == np.float32(s.max_penetration), i
    for i, (got, w) in enumerate(zip(arena.specimen_positions(), singles)):
        np.testing.assert_array_equal(got.view(np.uint32), w.download_positions().view(np.uint32),
                                      err_msg=f"specimen {i}")


def test_batched_generator_arena_runs(cuda_lib):
    from tangle_b200.device import DeviceWorld

    specimens = batched_specimens(count=6, seed=3, max_fibers=120)
    packeds = [PackedAssembly.from_assembly(a) for a in specimens]
    d = min(a.smallest_diameter() for a in specimens)
    cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * d, neighbor_capacity=256,
                             max_list_bytes=1 << 32).to_config(d)
    arena = DeviceWorld.arena(packeds, cfg.cell_list, cfg.max_step)
    status = arena.run_batch(cfg, 64)
    assert status.total_iterations > 0
    per_spec = arena.specimen_statuses(cfg)
    assert len(per_spec) == 6
    assert all(np.isfinite(s.max_penetration) for s in per_spec)


def test_arena_contact_lists_keep_every_specimen_bit_for_bit(cuda_lib):
    """The arena's contact lists (one contact skin for all specimens, one
    refresh flag) leave each specimen's positions those of the same
    specimen relaxed alone, across refreshes and rebuilds."""
    from tangle_b200.device import DeviceWorld

    assemblies = batched_specimens(count=6, seed=5, max_fibers=300)
    packs = [PackedAssembly.from_assembly(a) for a in assemblies]
    d = min(a.smallest_diameter() for a in assemblies)
    cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * d, neighbor_capacity=256,
                             max_list_bytes=1 << 30).to_config(d)
    fixed = RelaxationConfig(**{**cfg.__dict__, "force_full_iterations": True})
    arena = DeviceWorld.arena(packs, fixed.cell_list, fixed.max_step)
    assert arena.contact_list_info()["block"] > 0
    singles = [DeviceWorld(p, fixed.cell_list, fixed.max_step) for p in packs]
    for batch in (9, 23, 31):
        arena.run_batch(fixed, batch)
        for w in singles:
            w.run_batch(fixed, batch)
    assert arena.contact_list_info()["refreshes"] > 1
    for i, (got, w) in enumerate(zip(arena.specimen_positions(), singles)):
        np.testing.assert_array_equal(got.view(np.uint32), w.download_positions().view(np.uint32),
                                      err_msg=f"specimen {i}")
    # Gated batches: specimens stop at their own iteration (their slots then
    # read the Verlet lists), and the next batch resumes them.
    gated = RelaxationConfig(**{**cfg.__dict__, "penetration_tolerance": 0.05 * d})
    for batch in (40, 40, 40):
        arena.run_batch(gated, batch)
        last = [w.run_batch(gated, batch) for w in singles]
        statuses = arena.specimen_statuses(gated)
        assert [s.total_iterations for s in statuses] == [s.total_iterations for s in last]
        assert [s.converged for s in statuses] == [s.converged for s in last]
    for i, (got, w) in enumerate(zip(arena.specimen_positions(), singles)):
        np.testing.assert_array_equal(got.view(np.uint32), w.download_positions().view(np.uint32),
                                      err_msg=f"specimen {i} after the gated batches")
    for w in [arena] + singles:
        w.close()
