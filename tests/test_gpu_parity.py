"""Parity of the CUDA path with the oracle on identical inputs.

Contract (the tolerances are written in the asserts):
* grid sizing, cell assignments and sorted neighbor-pair sets: bit-exact;
* one contact pass (corrections and per-segment penetration): bit-exact;
* positions after a fixed iteration count: max |diff| <= 1e-5 * d (the
  stated tolerance), and in fact bit-exact: both sides round every f32
  operation identically, the arc cosine included (acos_f32);
* the admissibility verdict (converged, iteration count) identical.
"""

import numpy as np
import pytest

import fixtures as fx
from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import cpu_runnable_specimen, mid_size_specimen
from tangle_b200.settings import CellListConfig, RelaxationConfig, RelaxationSettings

pytestmark = pytest.mark.gpu


def worlds(assembly, max_step, cell_list=None, pin_ends=False):
    from oracle import OracleWorld
    from tangle_b200.device import DeviceWorld

    packed = PackedAssembly.from_assembly(assembly, pin_ends)
    cell_list = cell_list or CellListConfig()
    return OracleWorld(packed, cell_list, max_step), DeviceWorld(packed, cell_list, max_step), packed


def cases():
    d10 = 10.0e-6
    c1 = cpu_runnable_specimen()
    c1_cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * d10).to_config(c1.smallest_diameter())
    small = mid_size_specimen(scale=0.2, seed=3)
    small_cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * 7.0e-6, neighbor_capacity=256,
                                   max_list_bytes=1 << 30).to_config(small.smallest_diameter())
    small_overflow_cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * 7.0e-6,
                                            neighbor_capacity=16).to_config(small.smallest_diameter())
    mat = fx.dense_crossed_mat()
    mat_cfg = RelaxationConfig(penetration_tolerance=0.0, force_full_iterations=True, max_step=0.01)
    mat_cfg1 = RelaxationConfig(penetration_tolerance=0.0, force_full_iterations=True, max_step=0.01,
                                cell_list=CellListConfig(neighbor_capacity=1))
    zig = fx.pinned_zigzag()
    zig_cfg = RelaxationConfig(penetration_tolerance=1.0e-5, stretch_stiffness=0.0, bend_stiffness=0.0,
                               curvature_ratio_tolerance=1.0e-5, constraint_iterations=1,
                               curvature_cleanup_sweeps=1, max_step=0.02)
    walled = fx.hairpin()
    walled_cfg = RelaxationConfig(penetration_tolerance=1.0e-4, max_step=0.02)
    return [
        ("cpu_runnable", c1, c1_cfg, False, 10.0e-6),
        ("mid_size_scaled", small, small_cfg, False, 7.0e-6),
        ("mid_size_scaled_overflow", small, small_overflow_cfg, False, 7.0e-6),
        ("dense_mat", mat, mat_cfg, False, 0.2),
        ("dense_mat_overflow", mat, mat_cfg1, False, 0.2),
        ("zigzag", zig, zig_cfg, True, 0.01),
        ("hairpin_walls", walled, walled_cfg, False, 0.2),
    ]


CASES = cases()
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_sizing_cell_list_and_pair_sets_are_bit_exact(case, cuda_lib):
    name, assembly, cfg, pin, d = case
    orc, dev, packed = worlds(assembly, cfg.max_step, cfg.cell_list, pin)
    assert np.float32(dev.cell_size) == np.float32(orc.cell_size)
    assert dev.cell_dims == orc.cell_dims
    assert dev.neighbor_block == orc.neighbor_block
    assert np.float32(dev.neighbor_skin) == np.float32(orc.neighbor_skin)
    orc.debug_rebuild()
    dev.debug_rebuild()
    for a, b in zip(orc.debug_cell_list(), dev.debug_cell_list()):
        np.testing.assert_array_equal(a, b)
    oc, ol = orc.debug_neighbor_lists()
    dc, dl = dev.debug_neighbor_lists()
    np.testing.assert_array_equal(oc, dc)
    for s, (x, y) in enumerate(zip(ol, dl)):
        if x is None:
            assert y is None
        else:
            np.testing.assert_array_equal(x, y, err_msg=f"segment {s}")


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_contact_pass_is_bit_exact(case, cuda_lib):
    name, assembly, cfg, pin, d = case
    orc, dev, _ = worlds(assembly, cfg.max_step, cfg.cell_list, pin)
    oc, op = orc.debug_corrections(cfg)
    dc, dp = dev.debug_corrections(cfg)
    np.testing.assert_array_equal(op.view(np.uint32), dp.view(np.uint32))
    np.testing.assert_array_equal(oc.view(np.uint32), dc.view(np.uint32))


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_positions_after_fixed_iterations_agree(case, cuda_lib):
    name, assembly, cfg, pin, d = case
    orc, dev, packed = worlds(assembly, cfg.max_step, cfg.cell_list, pin)
    fixed = RelaxationConfig(**{**cfg.__dict__, "force_full_iterations": True})
    for batch in (7, 13):
        so = orc.run_batch(fixed, batch)
        sd = dev.run_batch(fixed, batch)
        assert (so.total_iterations, so.batch_iterations) == (sd.total_iterations, sd.batch_iterations)
    po, pd = orc.download_positions(), dev.download_positions()
    diff = float(np.abs(po.astype(np.float64) - pd.astype(np.float64)).max())
    assert diff <= 1.0e-5 * d, f"{name}: max |diff| {diff:.3e} > 1e-5 d"
    np.testing.assert_array_equal(po.view(np.uint32), pd.view(np.uint32))
    assert orc.neighbor_list_rebuilds() == dev.neighbor_list_rebuilds()


@pytest.mark.parametrize("period,ranked", [("1", "0"), ("1", "1"), ("0", "0")])
def test_positions_do_not_depend_on_the_update_order(period, ranked, cuda_lib, monkeypatch):
    """The grouped-lane update takes its fibers in creation order or ranked
    by the rounds of their curvature sweeps, whichever its timed epochs find
    faster (epochs of 16 launches on worlds of 4,096 fibers or more).
    TGL_UPDATE_ORDER_PERIOD=1 makes every launch of a small world an epoch
    (both orders in turn), TGL_UPDATE_ORDER_RANKED=1 ranks before every one,
    0 keeps the creation order: the positions stay bit-identical to the
    oracle's in every case."""
    monkeypatch.setenv("TGL_UPDATE_ORDER_PERIOD", period)
    monkeypatch.setenv("TGL_UPDATE_ORDER_RANKED", ranked)
    name, assembly, cfg, pin, d = CASES[IDS.index("mid_size_scaled")]
    orc, dev, _ = worlds(assembly, cfg.max_step, cfg.cell_list, pin)
    fixed = RelaxationConfig(**{**cfg.__dict__, "force_full_iterations": True})
    for batch in (5, 11, 16):
        so = orc.run_batch(fixed, batch)
        sd = dev.run_batch(fixed, batch)
        assert (so.total_iterations, so.batch_iterations) == (sd.total_iterations, sd.batch_iterations)
    np.testing.assert_array_equal(orc.download_positions().view(np.uint32), dev.download_positions().view(np.uint32))
    assert orc.neighbor_list_rebuilds() == dev.neighbor_list_rebuilds()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_admissibility_verdict_is_identical(case, cuda_lib):
    name, assembly, cfg, pin, d = case
    orc, dev, _ = worlds(assembly, cfg.max_step, cfg.cell_list, pin)
    budget = 400
    so = orc.run_batch(cfg, budget)
    sd = dev.run_batch(cfg, budget)
    assert so.converged == sd.converged
    assert so.total_iterations == sd.total_iterations
    assert so.cell_list_overflow == sd.cell_list_overflow
    for key in ("max_penetration", "max_curvature_ratio", "max_displacement"):
        a, b = getattr(so, key), getattr(sd, key)
        assert abs(a - b) <= 1.0e-5 * max(abs(a), abs(b), d), (key, a, b)


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_upload_rejects_non_finite_coordinates_and_keeps_the_state(bad, cuda_lib):
    """tgl_upload_positions checks the staged coordinates on the device
    before the world changes: a NaN or an infinity anywhere is refused with
    TGL_ERR_INVALID and the positions stay as they were."""
    from tangle_b200.device import DeviceWorld

    packed = PackedAssembly.from_assembly(cpu_runnable_specimen())
    dev = DeviceWorld(packed, CellListConfig(), 1.0e-6)
    before = dev.download_positions()
    for index in (0, before.size // 2, before.size - 1):
        xyz = before.copy()
        xyz[index] = bad
        with pytest.raises(ValueError, match="finite"):
            dev.upload_positions(xyz)
        np.testing.assert_array_equal(dev.download_positions().view(np.uint32), before.view(np.uint32))
    moved = before + np.float32(1.0e-7)
    dev.upload_positions(moved)
    np.testing.assert_array_equal(dev.download_positions().view(np.uint32), moved.view(np.uint32))
    dev.close()
