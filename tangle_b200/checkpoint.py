"""Restart checkpoints of a relaxation run.

Mirrors crates/tangle_checkpoint/src/lib.rs and the Python settings of
crates/tangle_python/src/checkpoint.rs for the plain relaxation path:

* `CheckpointSettings` has the reference's fields, defaults and validation
  (checkpoint.rs:30-105);
* a checkpoint holds the packed assembly with the current positions, cell,
  active fibers and curvature limits, the lifetime iteration count, the wall
  reactions and the installed layer and vertex targets
  (`DeviceWorldCheckpoint`, world.rs:280-304), plus the recipe's progress,
  and is written atomically (a temporary file renamed
  over the target, lib.rs:379-420) behind an 8-byte magic and a schema
  number that a load checks, with the case id (lib.rs:347-377);
* saves happen when the iteration count crosses a multiple of
  `interval_iterations` or the run ends (lib.rs:318-345).

The file body is this library's own (a NumPy archive), not the reference's
bincode payload, which serialises Rust types this library does not have.
"""

from __future__ import annotations

import dataclasses
import io
import os
import tempfile
import zipfile
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

import numpy as np

from .assembly import PackedAssembly
from .formation import LayerTargetCheckpoint, VertexTargetCheckpoint

MAGIC = b"TANGLEB2"
SCHEMA = 2

_PACKED_FIELDS = [f.name for f in dataclasses.fields(PackedAssembly)]


class CheckpointError(RuntimeError):
    """A checkpoint could not be read (lib.rs:140-190)."""


@dataclass
class DeviceWorldCheckpoint:
    """The persistent state of a device world (world.rs:280-304, plain path)."""

    packed: PackedAssembly
    total_iterations: int
    wall_reactions: Optional[np.ndarray] = None  # f32 [3V]
    layer_target: Optional[LayerTargetCheckpoint] = None
    vertex_target: Optional[VertexTargetCheckpoint] = None


@dataclass
class CheckpointSettings:
    """Periodic restart checkpoint and optional resume settings (_tangle.pyi:540-560)."""

    case_id: str
    path: Path
    interval_iterations: int = 500
    resume: bool = False
    resume_path: Optional[Path] = None
    resume_case_id: Optional[str] = None
    fresh_formation_on_resume: bool = False

    def __post_init__(self):
        self.path = Path(self.path)
        if self.resume_path is not None:
            self.resume_path = Path(self.resume_path)
        self.validate()

    def validate(self) -> None:
        """checkpoint.rs:76-105."""
        if not str(self.case_id).strip():
            raise ValueError("checkpoint case_id must not be empty")
        if int(self.interval_iterations) <= 0:
            raise ValueError("checkpoint interval_iterations must be positive")
        if self.resume_case_id is not None and not str(self.resume_case_id).strip():
            raise ValueError("resume_case_id must not be empty when supplied")

    def copy(self) -> "CheckpointSettings":
        return dataclasses.replace(self)

    def replace(self, **changes) -> "CheckpointSettings":
        return dataclasses.replace(self, **changes)


@dataclass
class CheckpointReport:
    """Saves made and the resume point (lib.rs:120-138)."""

    saves: int = 0
    last_saved_iteration: Optional[int] = None
    last_saved_bytes: Optional[int] = None
    resumed: bool = False
    resumed_iteration: Optional[int] = None


@dataclass
class RunCheckpoint:
    """What a recipe run saves: the world, and where the recipe stood."""

    case_id: str
    device: DeviceWorldCheckpoint
    operation: int  # index of the operation in progress
    operation_iterations: int  # iterations that operation had completed
    converged: bool


def encode(checkpoint: RunCheckpoint) -> bytes:
    packed = checkpoint.device.packed
    arrays = {f"packed_{name}": np.asarray(getattr(packed, name)) for name in _PACKED_FIELDS}
    arrays["case_id"] = np.frombuffer(checkpoint.case_id.encode("utf-8"), dtype=np.uint8)
    arrays["counters"] = np.array([checkpoint.device.total_iterations, checkpoint.operation,
                                   checkpoint.operation_iterations, int(checkpoint.converged)], dtype=np.uint64)
    device = checkpoint.device
    if device.wall_reactions is not None:
        arrays["wall_reactions"] = np.asarray(device.wall_reactions, dtype=np.float32)
    if device.layer_target is not None:
        t = device.layer_target
        arrays["layer_coordinates"] = np.asarray(t.coordinates, dtype=np.float32)
        arrays["layer_ints"] = np.array([t.axis, t.first_layer, t.last_layer], dtype=np.uint32)
        arrays["layer_gains"] = np.array([t.stiffness, t.max_translation], dtype=np.float32)
    if device.vertex_target is not None:
        t = device.vertex_target
        arrays["vertex_indices"] = np.asarray(t.indices, dtype=np.uint32)
        arrays["vertex_coordinates"] = np.asarray(t.coordinates, dtype=np.float32)
        arrays["vertex_commands"] = np.asarray(t.command_coordinates, dtype=np.float32)
        arrays["vertex_axis"] = np.array([t.axis], dtype=np.uint32)
        arrays["vertex_gains"] = np.array([t.stiffness, t.max_translation], dtype=np.float32)
    body = io.BytesIO()
    np.savez(body, **arrays)
    return MAGIC + SCHEMA.to_bytes(4, "little") + body.getvalue()


def decode(data: bytes, case_id: str) -> RunCheckpoint:
    """load_checkpoint (lib.rs:347-377): magic, schema, then the case id.
    Every failure to decode the body (a truncated file, a missing field, a
    malformed array) is a CheckpointError, as in the reference."""
    magic = data[: len(MAGIC)]
    schema = int.from_bytes(data[len(MAGIC): len(MAGIC) + 4], "little") if len(data) >= len(MAGIC) + 4 else 0
    if magic != MAGIC or schema != SCHEMA:
        raise CheckpointError(f"incompatible checkpoint schema: magic {magic!r}, schema {schema}")
    try:
        return _decode_body(data[len(MAGIC) + 4:], case_id)
    except CheckpointError:
        raise
    except (KeyError, ValueError, TypeError, EOFError, OSError, zipfile.BadZipFile) as error:
        raise CheckpointError(f"failed to decode checkpoint: {type(error).__name__}: {error}") from error


def _decode_body(body: bytes, case_id: str) -> RunCheckpoint:
    with np.load(io.BytesIO(body)) as archive:
        found = bytes(archive["case_id"]).decode("utf-8")
        if found != case_id:
            raise CheckpointError(f"checkpoint case mismatch: expected {case_id!r}, found {found!r}")
        packed = PackedAssembly(**{name: archive[f"packed_{name}"].copy() for name in _PACKED_FIELDS})
        total, operation, op_iterations, converged = (int(x) for x in archive["counters"])
        device = DeviceWorldCheckpoint(packed, total)
        if "wall_reactions" in archive:
            device.wall_reactions = archive["wall_reactions"].copy()
        if "layer_coordinates" in archive:
            axis, first, last = (int(x) for x in archive["layer_ints"])
            stiffness, max_translation = (float(x) for x in archive["layer_gains"])
            device.layer_target = LayerTargetCheckpoint(archive["layer_coordinates"].copy(), axis, first, last,
                                                        stiffness, max_translation)
        if "vertex_indices" in archive:
            stiffness, max_translation = (float(x) for x in archive["vertex_gains"])
            device.vertex_target = VertexTargetCheckpoint(archive["vertex_indices"].copy(),
                                                          archive["vertex_coordinates"].copy(),
                                                          archive["vertex_commands"].copy(),
                                                          int(archive["vertex_axis"][0]), stiffness, max_translation)
    return RunCheckpoint(found, device, operation, op_iterations, bool(converged))


def save(path: Path, checkpoint: RunCheckpoint) -> int:
    """Writes `checkpoint` to `path` atomically (lib.rs:392-420); returns its size."""
    data = encode(checkpoint)
    path = Path(path)
    if path.parent != Path(""):
        path.parent.mkdir(parents=True, exist_ok=True)
    fd, tmp = tempfile.mkstemp(prefix=path.name + ".", suffix=".tmp", dir=str(path.parent))
    try:
        with os.fdopen(fd, "wb") as fh:
            fh.write(data)
            fh.flush()
            os.fsync(fh.fileno())
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.unlink(tmp)
        raise
    return len(data)


def load(path: Path, case_id: str) -> RunCheckpoint:
    with open(path, "rb") as fh:
        return decode(fh.read(), case_id)


def crossed_interval(iteration: int, last_saved: Optional[int], interval: int) -> bool:
    """lib.rs:326-330."""
    if last_saved is None:
        return iteration >= interval
    return iteration // interval > last_saved // interval
