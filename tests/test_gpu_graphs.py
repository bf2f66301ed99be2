"""Batch graphs with the rebuild pipeline as a conditional node, looped on
the device.

A one-thread kernel sets an IF node's condition from the pending-rebuild
flag, so the eleven gated rebuild kernels launch only when a rebuild runs. The
alternative capture (`TGL_NO_CONDITIONAL_GRAPHS=1`, read when a world is
created) launches them every step and lets each return at once. Both must
give the same bits, and the launch count of the conditional graph must add
the eleven kernels only for the pipelines that ran.

By default the batch graph is one WHILE node over a single step: a kernel
sets the rebuild condition and the loop's own (another step while the gate
keeps the batch active and fewer than iterations + 1 steps have begun). The
unrolled capture (`TGL_NO_LOOP_GRAPHS=1`) holds iterations + 1 copies of
the step. Both give the same bits, statuses and rebuilds; the looped graph
stops launching once the gate has stopped the batch.
"""

import os

import numpy as np
import pytest

from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import cpu_runnable_specimen, mid_size_specimen
from tangle_b200.settings import CellListConfig, RelaxationConfig, RelaxationSettings

pytestmark = pytest.mark.gpu

REBUILD_KERNELS = 11


def make_world(packed, cell_list, max_step, conditional: bool, looped: bool = True):
    from tangle_b200.device import DeviceWorld

    saved = {k: os.environ.pop(k, None) for k in ("TGL_NO_CONDITIONAL_GRAPHS", "TGL_NO_LOOP_GRAPHS")}
    if not conditional:
        os.environ["TGL_NO_CONDITIONAL_GRAPHS"] = "1"
    if not looped:
        os.environ["TGL_NO_LOOP_GRAPHS"] = "1"
    try:
        return DeviceWorld(packed, cell_list, max_step)
    finally:
        for k, v in saved.items():
            os.environ.pop(k, None)
            if v is not None:
                os.environ[k] = v


def cases():
    c1 = cpu_runnable_specimen()
    c1_cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * 10.0e-6).to_config(c1.smallest_diameter())
    small = mid_size_specimen(scale=0.2, seed=5)
    small_cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * 7.0e-6, neighbor_capacity=256,
                                   max_list_bytes=1 << 30).to_config(small.smallest_diameter())
    return [("cpu_runnable", c1, c1_cfg), ("mid_size_scaled", small, small_cfg)]


CASES = cases()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_conditional_rebuild_matches_gated_launches(case, cuda_lib):
    name, assembly, cfg = case
    packed = PackedAssembly.from_assembly(assembly, False)
    fixed = RelaxationConfig(**{**cfg.__dict__, "force_full_iterations": True})
    cond = make_world(packed, cfg.cell_list, cfg.max_step, True)
    gated = make_world(packed, cfg.cell_list, cfg.max_step, False)
    for batch in (9, 31, 64):
        rebuilds = (cond.neighbor_list_rebuilds(), gated.neighbor_list_rebuilds())
        launches = (cond.kernel_launches, gated.kernel_launches)
        sc = cond.run_batch(fixed, batch)
        sg = gated.run_batch(fixed, batch)
        assert (sc.total_iterations, sc.batch_iterations) == (sg.total_iterations, sg.batch_iterations)
        new_rebuilds = cond.neighbor_list_rebuilds() - rebuilds[0]
        assert new_rebuilds == gated.neighbor_list_rebuilds() - rebuilds[1]
        # Per step the gated graph launches the eleven rebuild kernels, the
        # conditional one a condition kernel, plus the pipelines that ran.
        steps = batch + 1
        cond_launches = cond.kernel_launches - launches[0]
        gated_launches = gated.kernel_launches - launches[1]
        assert gated_launches - cond_launches == (REBUILD_KERNELS - 1) * steps - REBUILD_KERNELS * new_rebuilds, name
    assert cond.neighbor_list_rebuilds() > 0
    np.testing.assert_array_equal(cond.download_positions().view(np.uint32),
                                  gated.download_positions().view(np.uint32))


def test_conditional_graph_with_frequent_rebuilds(cuda_lib):
    """A neighbor skin of 0.05 fiber radii is passed by some vertex after
    almost every update (the oracle rebuilds 18 times in these 19 steps), so
    conditional bodies run back to back."""
    assembly = cpu_runnable_specimen()
    packed = PackedAssembly.from_assembly(assembly, False)
    cfg = RelaxationConfig(penetration_tolerance=0.0, force_full_iterations=True, max_step=2.0e-6)
    cell_list = CellListConfig(neighbor_skin_scale=0.05)
    cond = make_world(packed, cell_list, cfg.max_step, True)
    gated = make_world(packed, cell_list, cfg.max_step, False)
    launches = cond.kernel_launches, gated.kernel_launches
    before = cond.neighbor_list_rebuilds()
    for batch in (5, 12):
        cond.run_batch(cfg, batch)
        gated.run_batch(cfg, batch)
    assert cond.neighbor_list_rebuilds() == gated.neighbor_list_rebuilds()
    rebuilds = cond.neighbor_list_rebuilds() - before
    assert rebuilds >= 15
    steps = 5 + 1 + 12 + 1
    assert (gated.kernel_launches - launches[1]) - (cond.kernel_launches - launches[0]) == \
        (REBUILD_KERNELS - 1) * steps - REBUILD_KERNELS * rebuilds
    np.testing.assert_array_equal(cond.download_positions().view(np.uint32),
                                  gated.download_positions().view(np.uint32))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_looped_graph_matches_the_unrolled_one(case, cuda_lib):
    """Fixed-length batches and batches the gate stops early (the specimen
    converges): same statuses, rebuilds and bits; after the gate stops, the
    looped graph launches one more step and no further ones."""
    name, assembly, cfg = case
    packed = PackedAssembly.from_assembly(assembly, False)
    fixed = RelaxationConfig(**{**cfg.__dict__, "force_full_iterations": True})
    looped = make_world(packed, cfg.cell_list, cfg.max_step, True, True)
    unrolled = make_world(packed, cfg.cell_list, cfg.max_step, True, False)
    for config, batch in ((fixed, 9), (fixed, 40), (cfg, 128), (cfg, 128), (cfg, 64)):
        launches = (looped.kernel_launches, unrolled.kernel_launches)
        sl = looped.run_batch(config, batch)
        su = unrolled.run_batch(config, batch)
        assert sl == su, name
        assert looped.neighbor_list_rebuilds() == unrolled.neighbor_list_rebuilds()
        assert looped.kernel_launches - launches[0] <= unrolled.kernel_launches - launches[1]
        np.testing.assert_array_equal(looped.download_positions().view(np.uint32),
                                      unrolled.download_positions().view(np.uint32))
