"""Host-side logic that needs no GPU: packing, settings, generators, the
shared f32 arc cosine, and the C ABI's exported symbols."""

import ctypes
import math
import os
import re

import numpy as np
import pytest

import fixtures as fx
from tangle_b200.assembly import NONE, Cell, FiberAssembly, Material, PackedAssembly
from tangle_b200.generate import (SplitMix64, batched_specimens, cpu_runnable_specimen, mid_size_specimen,
                                  schladitz_axis_cosine_quantile)
from tangle_b200.settings import CellListConfig, RelaxationSettings

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_splitmix64_matches_the_published_sequence():
    """population.rs:795-812 is the standard SplitMix64 (first raw output for
    seed 0 is 0xE220A8397B1DCDAF); unit() keeps its top 53 bits."""
    rng = SplitMix64(0)
    u = rng.unit()
    assert u == float(0xE220A8397B1DCDAF >> 11) * 2.0 ** -53


def test_packing_follows_the_reference_layout():
    """packed.rs:200-270: consecutive segments, vertex_segments, interior-only
    curvature limits, f64 rest lengths cast to f32."""
    a = FiberAssembly(Cell([1.0] * 3, "xyz"))
    a.add_fiber([[0.1, 0.1, 0.1], [0.2, 0.1, 0.1], [0.3, 0.2, 0.1]], radius=0.01, min_bend_radius=0.5)
    a.add_fiber([[0.5, 0.5, 0.5], [0.5, 0.6, 0.5]], radius=0.02)
    p = PackedAssembly.from_assembly(a, pin_fiber_ends=True)
    assert p.segment_vertices.tolist() == [0, 1, 1, 2, 3, 4]
    assert p.segment_fibers.tolist() == [0, 0, 1]
    assert p.fiber_vertex_spans.tolist() == [0, 3, 3, 2]
    assert p.fiber_segment_spans.tolist() == [0, 2, 2, 1]
    assert p.vertex_segments.tolist() == [NONE, 0, 0, 1, 1, NONE, NONE, 2, 2, NONE]
    assert p.vertex_max_curvature.tolist() == [0.0, np.float32(2.0), 0.0, 0.0, 0.0]
    assert p.vertex_pinned.tolist() == [1, 0, 1, 1, 1]
    assert p.segment_rest_lengths[1] == np.float32(math.sqrt(0.1 ** 2 + 0.1 ** 2))
    assert p.cell_upper.tolist() == [1.0, 1.0, 1.0] and p.cell_periodic.tolist() == [1, 1, 1]


def test_settings_scale_unset_lengths_by_the_smallest_diameter():
    """settings.rs:474-499: 1 % and 10 % of the smallest diameter."""
    cfg = RelaxationSettings().to_config(10.0e-6)
    assert cfg.penetration_tolerance == np.float32(1.0e-7)
    assert cfg.max_step == np.float32(1.0e-6)
    cfg = RelaxationSettings(penetration_tolerance=2.0e-9, max_step=3.0e-7).to_config(10.0e-6)
    assert cfg.penetration_tolerance == np.float32(2.0e-9) and cfg.max_step == np.float32(3.0e-7)
    assert RelaxationSettings().to_config(None).max_step == np.float32(0.006)


@pytest.mark.parametrize("change, message", [
    ({"correction_fraction": 0.0}, "correction_fraction"),
    ({"stretch_stiffness": 1.5}, "stretch_stiffness"),
    ({"curvature_limit_safety_margin": 0.1}, "curvature_limit_safety_margin"),
    ({"constraint_iterations": 0}, "iteration and sweep counts"),
    ({"max_step": -1.0}, "max_step"),
    ({"cell_size_scale": 0.5}, "cell_size_scale"),
    ({"neighbor_skin_scale": -1.0}, "neighbor_skin_scale"),
    ({"neighbor_capacity": 0}, "neighbor_capacity"),
    ({"penetration_tolerance": float("nan")}, "penetration_tolerance"),
])
def test_settings_validation_matches_the_reference(change, message):
    """settings.rs:500-577 error messages."""
    with pytest.raises(ValueError, match=message):
        RelaxationSettings(**change).to_config(1.0e-5)


def test_settings_reject_what_the_plain_path_does_not_provide():
    with pytest.raises(ValueError):
        RelaxationSettings(backend="metal")
    with pytest.raises(ValueError, match="motion_model"):
        RelaxationSettings(motion_model="wobble")
    assert RelaxationSettings(motion_model="rigid_translation").to_config(1.0e-5).motion_code == 1
    assert RelaxationSettings().to_config(1.0e-5).motion_code == 0


def test_acos_f32_is_within_one_ulp():
    from oracle import _load

    lib = _load()
    lib.orc_acos_f32.argtypes = [ctypes.c_float]
    lib.orc_acos_f32.restype = ctypes.c_float
    xs = np.concatenate([np.linspace(-1.0, 1.0, 4001, dtype=np.float32),
                         (1.0 - np.logspace(-7, -1, 400)).astype(np.float32),
                         (-1.0 + np.logspace(-7, -1, 400)).astype(np.float32)])
    worst = 0.0
    for x in xs:
        exact = math.acos(float(x))
        got = lib.orc_acos_f32(float(x))
        worst = max(worst, abs(got - exact) / float(np.spacing(np.float32(exact))))
    assert worst <= 1.05


def test_cpu_runnable_specimen_shape():
    a = cpu_runnable_specimen()
    p = PackedAssembly.from_assembly(a)
    assert a.fiber_count == 40 and p.vertex_count == 1240 and p.segment_count == 1200
    assert np.allclose(p.segment_rest_lengths, 10.0e-6, rtol=1e-5)
    interior = p.vertex_max_curvature[p.vertex_max_curvature > 0]
    assert np.allclose(interior, 1.0 / 50.0e-6)


def test_mid_size_specimen_shape_and_volume_split():
    a = mid_size_specimen(scale=0.25)
    diameters = np.array([2 * f.radius for f in a.fibers])
    counts = {round(d * 1e6): int((np.round(diameters * 1e6) == round(d * 1e6)).sum()) for d in set(diameters)}
    assert set(counts) == {7, 19}
    volume_7 = counts[7] * 7.0 ** 2
    volume_19 = counts[19] * 19.0 ** 2
    assert abs(volume_7 / volume_19 - 1.0) < 0.1
    segs = {round(2 * f.radius * 1e6): f.placed.shape[0] - 1 for f in a.fibers}
    assert segs == {7: 107, 19: 39}


def test_schladitz_quantile_limits():
    """shape.rs:550-556: beta = 1 is isotropic (|cos| uniform)."""
    assert schladitz_axis_cosine_quantile(1.0, 0.3) == pytest.approx(0.3)
    assert schladitz_axis_cosine_quantile(0.3, 0.5) > 0.5  # axis-aligned for beta < 1
    assert schladitz_axis_cosine_quantile(1.0 / 0.3, 0.5) < 0.5  # in-plane for beta > 1


def test_batched_specimens_are_seeded_and_bounded():
    a = batched_specimens(count=3, seed=1, max_fibers=60)
    b = batched_specimens(count=3, seed=1, max_fibers=60)
    assert [x.fiber_count for x in a] == [x.fiber_count for x in b]
    for x in a:
        assert 40 <= x.fiber_count <= 60


def test_c_abi_library_loads_and_exports_every_declared_symbol():
    """The library loads without a GPU and exports what the header declares."""
    from tangle_b200.build import LIB, build
    from tangle_b200.device import EXPORTS

    build()
    lib = ctypes.CDLL(LIB)
    header = open(os.path.join(ROOT, "include", "tangle_cuda.h")).read()
    declared = set(re.findall(r"\b(tgl_[a-z0-9_]+)\s*\(", header))
    assert declared == set(EXPORTS)
    for name in declared:
        assert hasattr(lib, name), name


def test_no_fallback_when_the_library_is_missing(monkeypatch):
    import tangle_b200.device as device

    monkeypatch.setattr(device, "_lib", None)
    monkeypatch.setattr(device, "LIB_PATH", "/nonexistent/libtangle_cuda.so")
    with pytest.raises(RuntimeError, match="no fallback"):
        device.load_library()


@pytest.mark.parametrize("dims", [(1 << 21, 1 << 21, 1 << 22), (1 << 31, 1, 1), (1 << 16, 1 << 16, 1)],
                         ids=["wrapping_product", "axis_beyond_i32", "product"])
def test_grid_sizing_rejects_grids_whose_cell_count_would_overflow(dims):
    """The world's grid sizing (world.rs:410-415) rejects, before touching a
    GPU, a box whose per-axis cell counts overflow the 32-bit cell ids: an
    axis above 2^30, or a product above 2^31 -- also one that wraps to 0 in
    a 64-bit product (2^21 x 2^21 x 2^22 = 2^64)."""
    from oracle import OracleWorld
    from tangle_b200.device import DeviceWorld

    assembly = cpu_runnable_specimen()
    packed = PackedAssembly.from_assembly(assembly)
    cell = np.float32(OracleWorld(packed, CellListConfig(), 0.06 * 10e-6).cell_size)
    lower = np.zeros(3, dtype=np.float32)
    upper = np.array([cell * np.float32(n + 0.5) for n in dims], dtype=np.float32)
    # Each axis sizes to exactly the intended count (floor(extent / cell) in f32).
    assert [int(np.floor(np.float32(u) / cell)) for u in upper] == list(dims)
    packed.cell_lower[:] = lower
    packed.cell_upper[:] = upper
    with pytest.raises(Exception, match="cell grid too large"):
        OracleWorld(packed, CellListConfig(), 0.06 * 10e-6)
    with pytest.raises(Exception, match="cell grid too large"):
        DeviceWorld(packed, CellListConfig(), 0.06 * 10e-6)


def test_autotune_cache_keys_store_and_reload(tmp_path):
    """The autotuner's cache: one entry per (GPU, workload shape), written
    atomically and read back; a different shape or GPU misses."""
    from tangle_b200 import autotune as at

    shape = {"vertices": 10, "segments": 9, "cells": 27, "cell_dims": [3, 3, 3], "neighbor_block": 256,
             "specimens": 1, "contact_lists": True, "motion_model": "flexible"}
    key = at.workload_key("NVIDIA B200", shape)
    assert key == at.workload_key("NVIDIA B200", dict(reversed(list(shape.items()))))
    assert key != at.workload_key("NVIDIA H100", shape)
    assert key != at.workload_key("NVIDIA B200", {**shape, "vertices": 11})
    path = tmp_path / "sub" / "autotune.json"
    entry = {"params": {"lanes_per_fiber": 8, "contact_blocks_per_sm": 3, "build_chunk": 3072,
                        "contact_skin_fraction": 0.1}, "report": {"trials": 12}}
    at.store(path, key, entry)
    at.store(path, "other", {"params": {}})
    assert at.load(path)[key] == entry
    assert sorted(p.name for p in path.parent.iterdir()) == ["autotune.json"]  # no temporary left behind
    path.write_text("not json")
    assert at.load(path) == {}
    assert at.cache_path(str(path)) == path
