"""The FP64 contact-distance check on the CPU: the oracle's f32 contact pass
against the f64 restatement of the reference's host closest-point oracle
(world_tests.rs:1364-1485), on a scaled mid-size specimen.

* every sampled segment's maximum penetration (contact.rs:741-753) agrees
  with r1 + r2 - d64 over its listed neighbors within the stated f32 bound
  (16 units in the last place of the largest coordinate, `contact_f64.f32_bound`);
* every pair of a sampled segment within 0.999 (r1 + r2 + skin) in f64 is
  listed (world_tests.rs:1470-1479).
The same check runs on the CUDA pass at full size (test_gpu_full_size.py).
"""

import os

import numpy as np
import pytest

import contact_f64 as cf
from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import mid_size_specimen
from tangle_b200.settings import RelaxationSettings


@pytest.fixture(scope="module")
def scaled_pass():
    import oracle as orc

    orc.set_threads(os.cpu_count() or 1)
    assembly = mid_size_specimen(scale=0.25, seed=4)
    packed = PackedAssembly.from_assembly(assembly)
    d = assembly.smallest_diameter()
    cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * d, neighbor_capacity=256,
                             max_list_bytes=1 << 30).to_config(d)
    world = orc.OracleWorld(packed, cfg.cell_list, cfg.max_step)
    world.debug_rebuild()
    _, pen = world.debug_corrections(cfg)
    counts, lists = world.debug_neighbor_lists_raw()
    out = (packed, pen, counts, lists, world.neighbor_block, world.neighbor_skin, d)
    world.close()
    return out


def sample(pen, count=5000, seed=7):
    """Random segments plus as many segments in contact (the f64 check is
    sharpest where the penetration is positive)."""
    rng = np.random.default_rng(seed)
    hits = np.nonzero(pen > 0)[0]
    return np.unique(np.concatenate([rng.choice(pen.size, min(count, pen.size), replace=False),
                                     rng.choice(hits, min(count, hits.size), replace=False)]))


def test_oracle_contact_distances_agree_with_f64(scaled_pass):
    packed, pen, counts, lists, block, skin, d = scaled_pass
    report = cf.spot_check(packed, packed.positions, counts, lists, block, pen, sample(pen), skin)
    assert report["segments"] >= 5000 and report["in_contact"] >= 1000
    assert report["max_abs_error"] <= report["bound"], report
    assert report["bound"] <= 1.0e-3 * d  # the bound itself is far inside the 1e-3 d gate
    assert report["pairs_within_skin"] > 10 * report["segments"]
    assert report["missing"].shape[0] == 0, report["missing"][:10]


def test_f64_check_catches_a_planted_error(scaled_pass):
    """A penetration off by a few bounds, and a dropped list entry, are both
    caught (the mistakes are planted in a copy of the oracle's output)."""
    packed, pen, counts, lists, block, skin, d = scaled_pass
    segments = sample(pen, count=500)
    target = int(segments[np.argmax(pen[segments])])
    bad = pen.copy()
    bound = cf.f32_bound(packed.positions, np.asarray(packed.cell_upper) - np.asarray(packed.cell_lower))
    bad[target] = np.float32(bad[target] + 4.0 * bound)
    report = cf.spot_check(packed, packed.positions, counts, lists, block, bad, segments, skin)
    assert report["max_abs_error"] > report["bound"] and report["worst_segment"] == target
    dropped = lists.copy()
    n = int(counts[target])
    assert 0 < n <= block
    dropped_counts = counts.copy()
    dropped_counts[target] = n - 1  # the last (largest) neighbor disappears
    report = cf.spot_check(packed, packed.positions, dropped_counts, dropped, block, pen, segments, skin)
    assert report["missing"].shape[0] >= 1
