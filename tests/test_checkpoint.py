"""Restart checkpoints (tangle_checkpoint/src/lib.rs, world.rs:693-823).

CPU: settings validation, the file's magic/schema/case checks, an encode /
decode round trip and the save-interval rule. GPU: a world restored from a
checkpoint continues bit for bit where the original would have gone, with
its lifetime iteration count carried over, and a recipe run resumes from
its own checkpoint file.
"""

import numpy as np
import pytest

from tangle_b200 import checkpoint as ckpt
from tangle_b200.assembly import PackedAssembly
from tangle_b200.checkpoint import CheckpointSettings
from tangle_b200.generate import cpu_runnable_specimen
from tangle_b200.settings import RelaxationConfig, RelaxationSettings


def test_settings_defaults_and_validation(tmp_path):
    s = CheckpointSettings("case", tmp_path / "run.ckpt")
    assert (s.interval_iterations, s.resume, s.resume_path, s.resume_case_id, s.fresh_formation_on_resume) == (
        500, False, None, None, False)
    with pytest.raises(ValueError, match="case_id must not be empty"):
        CheckpointSettings("  ", tmp_path / "x")
    with pytest.raises(ValueError, match="interval_iterations must be positive"):
        CheckpointSettings("case", tmp_path / "x", interval_iterations=0)
    with pytest.raises(ValueError, match="resume_case_id must not be empty"):
        CheckpointSettings("case", tmp_path / "x", resume_case_id="")
    assert s.replace(interval_iterations=7).interval_iterations == 7


def _run_checkpoint(case_id="case"):
    packed = PackedAssembly.from_assembly(cpu_runnable_specimen())
    packed.positions = packed.positions + np.float32(1.0e-6)
    return ckpt.RunCheckpoint(case_id, ckpt.DeviceWorldCheckpoint(packed, 1234), 2, 56, True)


def test_file_round_trip_and_atomic_write(tmp_path):
    original = _run_checkpoint()
    path = tmp_path / "sub" / "run.ckpt"
    size = ckpt.save(path, original)
    assert path.stat().st_size == size
    assert [p.name for p in path.parent.iterdir()] == ["run.ckpt"]  # no temporary left behind
    loaded = ckpt.load(path, "case")
    assert (loaded.device.total_iterations, loaded.operation, loaded.operation_iterations, loaded.converged) == (
        1234, 2, 56, True)
    for name in ("positions", "intrinsic_positions", "segment_vertices", "vertex_segments", "cell_periodic"):
        a, b = getattr(original.device.packed, name), getattr(loaded.device.packed, name)
        assert a.dtype == b.dtype
        np.testing.assert_array_equal(a, b)


def test_load_rejects_other_cases_and_schemas(tmp_path):
    path = tmp_path / "run.ckpt"
    ckpt.save(path, _run_checkpoint("first"))
    with pytest.raises(ckpt.CheckpointError, match="case mismatch"):
        ckpt.load(path, "second")
    data = bytearray(path.read_bytes())
    data[8] ^= 0xFF  # schema
    path.write_bytes(bytes(data))
    with pytest.raises(ckpt.CheckpointError, match="incompatible checkpoint schema"):
        ckpt.load(path, "first")
    path.write_bytes(b"TANGLE01" + b"\x04\x00\x00\x00")  # the reference's own header
    with pytest.raises(ckpt.CheckpointError, match="incompatible"):
        ckpt.load(path, "first")


def test_save_interval_rule():
    # lib.rs:326-330: the first save once `interval` is reached, then one per
    # crossed multiple.
    assert not ckpt.crossed_interval(499, None, 500)
    assert ckpt.crossed_interval(500, None, 500)
    assert not ckpt.crossed_interval(999, 500, 500)
    assert ckpt.crossed_interval(1000, 999, 500)
    assert ckpt.crossed_interval(1600, 900, 500)


@pytest.mark.gpu
def test_restored_world_continues_bit_for_bit(cuda_lib):
    from tangle_b200.device import DeviceWorld

    assembly = cpu_runnable_specimen(seed=3)
    config = RelaxationSettings(penetration_tolerance=1.0e-3 * 10.0e-6).to_config(assembly.smallest_diameter())
    fixed = RelaxationConfig(**{**config.__dict__, "force_full_iterations": True})
    packed = PackedAssembly.from_assembly(assembly)
    straight = DeviceWorld.upload(config, packed)
    straight.run_batch(fixed, 11)
    straight.run_batch(fixed, 9)
    halfway = DeviceWorld.upload(config, packed)
    halfway.run_batch(fixed, 11)
    state = halfway.checkpoint()
    assert state.total_iterations == 11
    np.testing.assert_array_equal(state.packed.positions, halfway.download_positions())
    halfway.close()
    restored = DeviceWorld.restore(config, state)
    status = restored.run_batch(fixed, 9)
    assert status.total_iterations == 20 and status.batch_iterations == 9
    np.testing.assert_array_equal(restored.download_positions().view(np.uint32),
                                  straight.download_positions().view(np.uint32))


@pytest.mark.gpu
def test_recipe_saves_and_resumes(cuda_lib, tmp_path):
    from tangle_b200.assembly import Cell
    from tangle_b200.recipe import Recipe

    def recipe():
        r = Recipe(Cell([300.0e-6] * 3, periodic="xyz"))
        r.insert(cpu_runnable_specimen(seed=4))
        r.relax_for(60)
        return r

    settings = RelaxationSettings(iterations_per_batch=16, penetration_tolerance=1.0e-8)
    path = tmp_path / "run.ckpt"
    full = recipe().run(settings, checkpoint=CheckpointSettings("c1", path, interval_iterations=32))
    # Saves at 32 (crossing) and at the end (60).
    assert full.checkpoint_saves == 2 and full.last_checkpoint_iteration == 60
    assert full.last_checkpoint_bytes == path.stat().st_size
    saved = ckpt.load(path, "c1")
    assert saved.device.total_iterations == 60
    resumed = recipe().run(settings, checkpoint=CheckpointSettings("c1", path, resume=True,
                                                                   interval_iterations=32))
    assert resumed.resumed and resumed.resumed_iteration == 60
    # The recipe had finished: nothing more to run.
    assert resumed.iterations == 60
    np.testing.assert_array_equal(np.asarray(resumed.centerlines()), np.asarray(full.centerlines()))


@pytest.mark.gpu
def test_recipe_activates_inserted_fibers_step_by_step(cuda_lib):
    """kernels.rs:164-221: fibers inserted after a relaxation step take no
    part in it; the relaxation of the earlier fibers is that of a world
    holding only them, and the lifetime iteration count runs on."""
    from tangle_b200.assembly import Cell
    from tangle_b200.device import DeviceWorld
    from tangle_b200.recipe import Recipe

    cell = Cell([300.0e-6] * 3, periodic="xyz")
    first, second = cpu_runnable_specimen(seed=21), cpu_runnable_specimen(seed=22)
    settings = RelaxationSettings(iterations_per_batch=16, penetration_tolerance=1.0e-8)
    config = settings.to_config(first.smallest_diameter())

    r = Recipe(cell)
    r.insert(first)
    r.relax_for(20)
    r.insert(second)
    staged = r.run(settings)
    alone = DeviceWorld.upload(config, PackedAssembly.from_assembly(first))
    fixed = RelaxationConfig(**{**config.__dict__, "force_full_iterations": True})
    alone.run_batch(fixed, 16)
    alone.run_batch(fixed, 4)
    got = np.concatenate([np.asarray(c, dtype=np.float32).ravel() for c in staged.centerlines()[:first.fiber_count]])
    np.testing.assert_array_equal(got.view(np.uint32), alone.download_positions().view(np.uint32))
    # The later fibers took no part: they come back as uploaded (f32).
    for fiber, placed in zip(staged.assembly.fibers[first.fiber_count:], second.fibers):
        np.testing.assert_array_equal(fiber.placed, placed.placed.astype(np.float32).astype(np.float64))
    assert staged.iterations == 20

    r.relax_for(10)
    both = r.run(settings)
    assert both.iterations == 30
    moved = [not np.array_equal(f.placed, p.placed) for f, p in zip(both.assembly.fibers[first.fiber_count:],
                                                                    second.fibers)]
    assert any(moved)


def test_truncated_or_incomplete_files_raise_checkpoint_error(tmp_path):
    """Every decode failure is a CheckpointError (lib.rs:347-377 maps them all)."""
    import io as _io

    path = tmp_path / "run.ckpt"
    ckpt.save(path, _run_checkpoint("case"))
    data = path.read_bytes()
    header = len(ckpt.MAGIC) + 4
    for cut in (header, header + 10, len(data) // 2, len(data) - 1):
        path.write_bytes(data[:cut])
        with pytest.raises(ckpt.CheckpointError, match="failed to decode"):
            ckpt.load(path, "case")
    # A well-formed archive that lacks the fields.
    body = _io.BytesIO()
    np.savez(body, case_id=np.frombuffer(b"case", dtype=np.uint8))
    path.write_bytes(data[:header] + body.getvalue())
    with pytest.raises(ckpt.CheckpointError, match="failed to decode"):
        ckpt.load(path, "case")
