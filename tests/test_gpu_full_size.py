"""Parity on the bench's own configuration: the full mid-size specimen.

The bench reports throughput on the periodic 2 mm cube of 20,000 wavy
fibers (1,997,480 nodes, 1,977,480 segments, seed 1, neighbor capacity 256,
list cap 8 GiB). This module compares the CUDA path with the oracle on that
exact input, at full size:

* grid sizing, cell assignments (counts, offsets, slot order) and the
  sorted Verlet pair sets: bit-exact;
* one contact pass (corrections and per-segment maximum penetration):
  bit-exact;
* positions after 8 iterations: max |diff| <= 1e-5 d (the stated
  tolerance), and bit-identical; iteration count, rebuilds and the
  admissibility verdict identical;
* contact distances against an f64 restatement of the reference's host
  closest-point oracle (world_tests.rs:1364-1485): on >= 10,000 sampled
  segments (5,000 random, 5,000 in contact), the CUDA pass's maximum
  penetration is within the stated f32 bound of r1 + r2 - d64
  (`contact_f64.f32_bound`: 16 units in the last place of the largest
  coordinate plus a box length) and inside 1e-3 d, and every pair within 0.999 (r1 + r2 + skin) in f64 is in the
  CUDA lists.
"""

import os

import numpy as np
import pytest

import contact_f64 as cf
from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import mid_size_specimen
from tangle_b200.settings import RelaxationConfig, RelaxationSettings

pytestmark = pytest.mark.gpu

ITERATIONS = 8


def bench_config(assembly):
    """bench.py's settings for the mid-size workload."""
    d = assembly.smallest_diameter()
    settings = RelaxationSettings(penetration_tolerance=1.0e-3 * d, neighbor_capacity=256, max_list_bytes=8 << 30,
                                  iterations_per_batch=128, max_iterations=100000)
    return settings.to_config(d), d


@pytest.fixture(scope="module")
def full_size(cuda_lib):
    import oracle as orc
    from tangle_b200.device import DeviceWorld

    orc.set_threads(os.cpu_count() or 1)
    assembly = mid_size_specimen(seed=1)
    packed = PackedAssembly.from_assembly(assembly)
    cfg, d = bench_config(assembly)
    out = {"packed": packed, "cfg": cfg, "d": d}
    dev = DeviceWorld(packed, cfg.cell_list, cfg.max_step)
    ref = orc.OracleWorld(packed, cfg.cell_list, cfg.max_step)
    out["sizing"] = [(w.cell_size, w.cell_dims, w.neighbor_block, w.neighbor_skin) for w in (ref, dev)]
    ref.debug_rebuild()
    dev.debug_rebuild()
    out["cell_lists"] = (ref.debug_cell_list(), dev.debug_cell_list())
    out["lists"] = (ref.debug_neighbor_lists_raw(), dev.debug_neighbor_lists_raw())
    out["block"] = dev.neighbor_block
    out["skin"] = dev.neighbor_skin
    out["contact"] = (ref.debug_corrections(cfg), dev.debug_corrections(cfg))
    fixed = RelaxationConfig(**{**cfg.__dict__, "force_full_iterations": True})
    out["status"] = (ref.run_batch(fixed, ITERATIONS), dev.run_batch(fixed, ITERATIONS))
    out["positions"] = (ref.download_positions(), dev.download_positions())
    out["rebuilds"] = (ref.neighbor_list_rebuilds(), dev.neighbor_list_rebuilds())
    ref.close()
    dev.close()
    return out


def test_full_size_sizing_and_cell_list_are_bit_exact(full_size):
    (rs, rd, rb, rk), (ds, dd, db, dk) = full_size["sizing"]
    assert full_size["packed"].vertex_count == 1997480
    assert np.float32(rs) == np.float32(ds) and rd == dd and rb == db and np.float32(rk) == np.float32(dk)
    for a, b in zip(*full_size["cell_lists"]):
        np.testing.assert_array_equal(a, b)


def test_full_size_pair_sets_are_bit_exact(full_size):
    (rc, rl), (dc, dl) = full_size["lists"]
    block = full_size["block"]
    np.testing.assert_array_equal(rc, dc)
    assert int(rc.max()) <= block  # no overflowed segment: every list is compared
    valid = np.arange(block, dtype=np.uint32)[None, :] < rc[:, None]
    np.testing.assert_array_equal(rl.reshape(-1, block)[valid], dl.reshape(-1, block)[valid])


def test_full_size_contact_pass_is_bit_exact(full_size):
    (rc, rp), (dc, dp) = full_size["contact"]
    assert int((dp > 0).sum()) > 100000  # the initial packing overlaps widely
    np.testing.assert_array_equal(rp.view(np.uint32), dp.view(np.uint32))
    np.testing.assert_array_equal(rc.view(np.uint32), dc.view(np.uint32))


def test_full_size_positions_after_fixed_iterations_agree(full_size):
    po, pd = full_size["positions"]
    so, sd = full_size["status"]
    d = full_size["d"]
    diff = float(np.abs(po.astype(np.float64) - pd.astype(np.float64)).max())
    assert diff <= 1.0e-5 * d, f"max |diff| {diff:.3e} > 1e-5 d"
    np.testing.assert_array_equal(po.view(np.uint32), pd.view(np.uint32))
    assert (so.total_iterations, so.batch_iterations) == (sd.total_iterations, sd.batch_iterations) == (
        ITERATIONS, ITERATIONS)
    assert so.converged == sd.converged
    assert full_size["rebuilds"][0] == full_size["rebuilds"][1]
    for key in ("max_penetration", "max_curvature_ratio", "max_displacement"):
        a, b = getattr(so, key), getattr(sd, key)
        assert abs(a - b) <= 1.0e-5 * max(abs(a), abs(b), d), (key, a, b)


def test_full_size_contact_distances_agree_with_f64(full_size):
    packed = full_size["packed"]
    (_, pen) = full_size["contact"][1]
    counts, lists = full_size["lists"][1]
    rng = np.random.default_rng(11)
    hits = np.nonzero(pen > 0)[0]
    segments = np.unique(np.concatenate([rng.choice(pen.size, 5000, replace=False),
                                         rng.choice(hits, 5000, replace=False)]))
    report = cf.spot_check(packed, packed.positions, counts, lists, full_size["block"], pen, segments,
                           full_size["skin"])
    assert report["segments"] >= 10000 - 100  # overlap of the two draws only
    assert report["in_contact"] >= 5000
    assert report["max_abs_error"] <= report["bound"], report
    # Unwrapped coordinates reach about 6 mm here, so the bound is about
    # 1.06e-3 d; the errors themselves must also sit inside the gate's 1e-3 d.
    assert report["max_abs_error"] <= 1.0e-3 * full_size["d"], report
    assert report["missing"].shape[0] == 0, report["missing"][:10]
