"""Contact lists: the second list level under the Verlet lists changes nothing.

The contact pass reads, per cell-list slot, the Verlet-list entries within a
contact skin of touching at a snapshot, until a vertex moves half that skin
or the Verlet lists are rebuilt. These tests run the relaxation with contact
lists off, with a tiny contact skin (a refresh nearly every iteration) and
with the whole neighbor skin, and require the oracle's positions bit for bit
each time; and they check that every contact list is an ascending
sub-sequence of its segment's Verlet list.
"""

import numpy as np
import pytest

import fixtures as fx
from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import cpu_runnable_specimen, mid_size_specimen
from tangle_b200.settings import CellListConfig, RelaxationConfig, RelaxationSettings

pytestmark = pytest.mark.gpu


def specimens():
    c1 = cpu_runnable_specimen(seed=2)
    c1_cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * 10.0e-6).to_config(c1.smallest_diameter())
    small = mid_size_specimen(scale=0.2, seed=4)
    small_cfg = RelaxationSettings(penetration_tolerance=1.0e-3 * 7.0e-6, neighbor_capacity=256,
                                   max_list_bytes=1 << 30).to_config(small.smallest_diameter())
    mat = fx.dense_crossed_mat()
    mat_cfg = RelaxationConfig(penetration_tolerance=0.0, force_full_iterations=True, max_step=0.01)
    return [("cpu_runnable", c1, c1_cfg), ("mid_size_scaled", small, small_cfg), ("dense_mat", mat, mat_cfg)]


SPECIMENS = specimens()


def run_pair(assembly, cfg, iterations=(7, 13)):
    from oracle import OracleWorld
    from tangle_b200.device import DeviceWorld

    packed = PackedAssembly.from_assembly(assembly)
    orc = OracleWorld(packed, cfg.cell_list, cfg.max_step)
    dev = DeviceWorld(packed, cfg.cell_list, cfg.max_step)
    fixed = RelaxationConfig(**{**cfg.__dict__, "force_full_iterations": True})
    for batch in iterations:
        so = orc.run_batch(fixed, batch)
        sd = dev.run_batch(fixed, batch)
        assert (so.total_iterations, so.batch_iterations) == (sd.total_iterations, sd.batch_iterations)
    return orc, dev


@pytest.mark.parametrize("fraction", ["0", "0.02", "0.25", "1"])
@pytest.mark.parametrize("case", SPECIMENS, ids=[c[0] for c in SPECIMENS])
def test_positions_match_the_oracle_for_any_contact_skin(case, fraction, cuda_lib, monkeypatch):
    name, assembly, cfg = case
    monkeypatch.setenv("TGL_CONTACT_SKIN", fraction)
    orc, dev = run_pair(assembly, cfg)
    info = dev.contact_list_info()
    if fraction == "0":
        assert info["skin"] == 0.0 and info["block"] == 0
    else:
        assert np.float32(info["skin"]) == np.float32(float(fraction) * np.float32(dev.neighbor_skin))
        assert info["refreshes"] >= dev.neighbor_list_rebuilds() >= 1
    po, pd = orc.download_positions(), dev.download_positions()
    np.testing.assert_array_equal(po.view(np.uint32), pd.view(np.uint32), err_msg=f"{name} at {fraction}")
    assert orc.neighbor_list_rebuilds() == dev.neighbor_list_rebuilds()


@pytest.mark.parametrize("case", SPECIMENS, ids=[c[0] for c in SPECIMENS])
def test_contact_lists_are_ordered_sub_sequences_of_the_verlet_lists(case, cuda_lib, monkeypatch):
    name, assembly, cfg = case
    monkeypatch.setenv("TGL_CONTACT_SKIN", "0.25")
    _, dev = run_pair(assembly, cfg, iterations=(5,))
    _, _, slot_segment = dev.debug_cell_list()
    verlet_counts, verlet = dev.debug_neighbor_lists()
    counts, lists = dev.debug_contact_lists()
    block = dev.contact_list_info()["block"]
    checked = 0
    for slot, entries in enumerate(lists):
        segment = int(slot_segment[slot])
        full = verlet[segment]
        if full is None or entries is None:
            continue
        assert counts[slot] == len(entries) <= verlet_counts[segment]
        assert np.all(np.diff(entries.astype(np.int64)) > 0), f"slot {slot} not ascending"
        assert np.isin(entries, full).all(), f"slot {slot} holds entries outside its Verlet list"
        checked += 1
    assert checked > 0
    # The contact lists are shorter than the Verlet lists they filter, and a
    # batch's lists fit its chunk of 32 * block entries.
    chunked = np.array([0 if entries is None else len(entries) for entries in lists], dtype=np.int64)
    assert chunked.sum() <= verlet_counts.astype(np.int64).sum()
    padded = np.zeros((len(lists) + 31) // 32 * 32, dtype=np.int64)
    padded[:len(lists)] = chunked
    assert padded.reshape(-1, 32).sum(axis=1).max() <= 32 * block


def test_a_full_chunk_sends_its_last_lists_to_the_verlet_lists(cuda_lib, monkeypatch):
    """With the whole neighbor skin as contact skin the lists nearly equal
    the Verlet lists (about 41 entries a segment), more than a batch's chunk
    of 32 * 32 entries holds: the slots whose lists run past the chunk read
    their Verlet lists, and the positions stay the oracle's bit for bit."""
    name, assembly, cfg = SPECIMENS[1]
    monkeypatch.setenv("TGL_CONTACT_SKIN", "1")
    orc, dev = run_pair(assembly, cfg, iterations=(3, 5))
    counts, lists = dev.debug_contact_lists()
    on_verlet = sum(1 for entries in lists if entries is None)
    assert on_verlet > 0
    assert any(entries is not None and len(entries) > 0 for entries in lists)
    np.testing.assert_array_equal(orc.download_positions().view(np.uint32), dev.download_positions().view(np.uint32))
