"""Formation hooks of the resident world: staged activation, layer and vertex
targets, cell compaction and its metrics.

These are the `DeviceFiberWorld` methods the reference's formation recipes
drive between relaxation batches (crates/tangle_relax/src/device/world.rs:
1723-2194, through the `DeviceWorld` seam of plugin.rs:639-880), with the
reference's names, argument meanings and validation (its `assert!`s raise
`ValueError` here). `FormationHooks` holds the shared front end; a world
class supplies the low-level `_fh_*` calls (the CUDA library for
`DeviceWorld`).

* `activate_formation_step(k)` makes the fibers whose formation step is at
  most k take part and freezes the others (kernels.rs:164-221).
* `apply_layer_targets` / `apply_single_layer_target` install a layer target
  that pulls each targeted fiber's mean coordinate toward its layer's target
  once at once and then at the end of every update step, until
  `clear_layer_targets` (kernels.rs:538-581).
* `apply_vertex_displacement_targets` installs needle-like targets on chosen
  vertices (kernels.rs:583-634); `clear_vertex_targets` releases them.
* `formation_target_error` measures both targets' residuals.
* `compact_cell` shrinks the cell with one of three kinematics
  (kernels.rs:712-818); `compaction_metrics` and `wall_face_pressures` read
  the pressures and penalty energies (kernels.rs:820-923).
"""

from __future__ import annotations

import enum
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

NONE = 0xFFFFFFFF


class CompactionKinematics(enum.IntEnum):
    """How active fibers follow a shrinking cell (world.rs CompactionKinematics)."""

    RIGID_FIBER_CENTERS = 0  # each fiber keeps its centre's fractional position
    MOVING_WALLS = 1  # vertices projected inside the new walls
    AFFINE_VERTICES = 2  # every vertex scaled with the cell


@dataclass
class CompactionEnergyModel:
    """Stiffnesses of the penalty energies (world.rs CompactionEnergyModel)."""

    contact_stiffness: float = 1.0
    stretch_stiffness: float = 1.0
    bending_stiffness: float = 1.0


@dataclass
class CompactionMetrics:
    """Directional pressures and penalty energies (world.rs CompactionMetrics)."""

    pressure: Tuple[float, float, float]
    contact_energy: float
    stretch_energy: float
    bending_energy: float
    total_energy: float


@dataclass
class FormationTargetError:
    """Largest layer-centre and targeted-vertex residuals; None where no
    target is installed (world.rs FormationTargetError)."""

    layer: Optional[float] = None
    vertex: Optional[float] = None


@dataclass
class LayerTargetCheckpoint:
    """An installed layer target (world.rs:246-262)."""

    coordinates: np.ndarray
    axis: int
    first_layer: int
    last_layer: int
    stiffness: float
    max_translation: float


@dataclass
class VertexTargetCheckpoint:
    """Installed vertex targets with their commanded coordinates (world.rs:264-279)."""

    indices: np.ndarray
    coordinates: np.ndarray
    command_coordinates: np.ndarray
    axis: int
    stiffness: float
    max_translation: float


def _check_gains(stiffness: float, max_translation: float) -> None:
    if not (0.0 < stiffness <= 1.0):
        raise ValueError("stiffness must be in (0, 1]")
    if not (max_translation > 0.0):
        raise ValueError("max_translation must be positive")


class FormationHooks:
    """The formation methods of a single resident world.

    A world class sets `_packed` (its PackedAssembly) and implements
    `_fh_set_active`, `_fh_set_layer_targets`, `_fh_set_vertex_targets`,
    `_fh_vertex_target_state`, `_fh_target_errors`, `_fh_compact`,
    `_fh_cell_bounds`, `_fh_metrics`, `_fh_wall_reactions`,
    `_fh_set_wall_reactions` and `_fh_set_fiber_curvatures`.
    """

    _layer_state: Optional[LayerTargetCheckpoint] = None
    _vertex_indices: Optional[np.ndarray] = None
    _vertex_gains: Optional[Tuple[int, float, float]] = None
    _last_metrics: Optional[np.ndarray] = None
    _fiber_active: Optional[np.ndarray] = None
    _vertex_max_curvature: Optional[np.ndarray] = None

    # ---- staged activation

    def activate_formation_step(self, maximum_step: int) -> Tuple[int, int]:
        """world.rs:2139-2183: every fiber assigned to a step up to
        `maximum_step` takes part in later batches, the rest freeze; returns
        the active segment and vertex counts."""
        flags = (np.asarray(self._packed.fiber_formation_steps) <= int(maximum_step)).astype(np.uint8)
        return self.set_active_fibers(flags)

    def set_active_fibers(self, active: Sequence[bool]) -> Tuple[int, int]:
        """The fibers with a true flag take part; the others freeze."""
        flags = np.ascontiguousarray(np.asarray(active).astype(np.uint8))
        if flags.size != self._packed.fiber_count:
            raise ValueError("active flags need one entry per fiber")
        counts = self._fh_set_active(flags)
        self._fiber_active = flags.astype(np.uint32)
        return counts

    @property
    def fiber_active(self) -> np.ndarray:
        if self._fiber_active is None:
            return np.asarray(self._packed.fiber_active, dtype=np.uint32).copy()
        return self._fiber_active.copy()

    def unpack_positions(self, positions, assembly) -> None:
        """Installs downloaded positions in `assembly` and keeps only the
        active fibers (world.rs unpack_positions after staged activation)."""
        self._packed.unpack_positions(positions, assembly)
        keep = self.fiber_active
        assembly.fibers = [f for f, on in zip(assembly.fibers, keep) if on]

    # ---- layer targets

    def apply_layer_targets(self, axis: int, targets: Sequence[float], stiffness: float,
                            max_translation: float) -> None:
        """world.rs:1721-1740: a persistent target for every layer, applied
        once now and after every update step."""
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        if targets.size == 0:
            raise ValueError("layer targets must not be empty")
        self._layer_range(axis, targets, 0, targets.size - 1, stiffness, max_translation, True)

    def apply_single_layer_target(self, axis: int, targets: Sequence[float], layer: int, stiffness: float,
                                  max_translation: float) -> None:
        """world.rs:1742-1755: a target for one newly deposited layer, leaving
        the already relaxed stack free."""
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        if not 0 <= int(layer) < targets.size:
            raise ValueError("layer must index the targets")
        self._layer_range(axis, targets, int(layer), int(layer), stiffness, max_translation, True)

    def _layer_range(self, axis, targets, first, last, stiffness, max_translation, apply_now) -> None:
        if axis not in (0, 1, 2):
            raise ValueError("axis must be 0, 1 or 2")
        _check_gains(float(stiffness), float(max_translation))
        layers = np.ascontiguousarray(self._packed.fiber_formation_layers, dtype=np.uint32)
        self._fh_set_layer_targets(int(axis), targets, layers, first, last, float(stiffness),
                                   float(max_translation), apply_now)
        self._layer_state = LayerTargetCheckpoint(targets.copy(), int(axis), first, last, float(stiffness),
                                                  float(max_translation))

    def clear_layer_targets(self) -> None:
        """world.rs:1806-1810."""
        self._fh_set_layer_targets(0, None, None, 0, 0, 0.0, 0.0, False)
        self._layer_state = None

    # ---- vertex targets

    def apply_vertex_displacement_targets(self, axis: int, vertex_indices: Sequence[int], displacement: float,
                                          stiffness: float, max_translation: float) -> None:
        """world.rs:1811-1859: each listed vertex's target is its current
        coordinate plus `displacement`; at the end of every update step it is
        set to a commanded coordinate that advances toward the target."""
        indices = np.ascontiguousarray(vertex_indices, dtype=np.uint32)
        if axis not in (0, 1, 2):
            raise ValueError("axis must be 0, 1 or 2")
        if indices.size == 0:
            raise ValueError("vertex targets must not be empty")
        if np.any(indices >= self._packed.vertex_count):
            raise ValueError("vertex target index out of range")
        if not (np.isfinite(displacement) and displacement != 0.0):
            raise ValueError("displacement must be finite and non-zero")
        _check_gains(float(stiffness), float(max_translation))
        self._fh_set_vertex_targets(int(axis), indices, float(displacement), float(stiffness),
                                    float(max_translation), None, None)
        self._vertex_indices = indices.copy()
        self._vertex_gains = (int(axis), float(stiffness), float(max_translation))

    def clear_vertex_targets(self) -> None:
        """world.rs:1861-1863."""
        self._fh_set_vertex_targets(0, None, 0.0, 0.0, 0.0, None, None)
        self._vertex_indices = None
        self._vertex_gains = None

    def vertex_target_checkpoint(self) -> Optional[VertexTargetCheckpoint]:
        if self._vertex_indices is None:
            return None
        coordinates, commands = self._fh_vertex_target_state(self._vertex_indices.size)
        axis, stiffness, max_translation = self._vertex_gains
        return VertexTargetCheckpoint(self._vertex_indices.copy(), coordinates, commands, axis, stiffness,
                                      max_translation)

    def layer_target_checkpoint(self) -> Optional[LayerTargetCheckpoint]:
        return self._layer_state

    def formation_target_error(self) -> FormationTargetError:
        """world.rs:1865-1929."""
        layer, has_layer, vertex, has_vertex = self._fh_target_errors()
        return FormationTargetError(layer if has_layer else None, vertex if has_vertex else None)

    # ---- compaction

    def compact_cell(self, new_lower: Sequence[float], new_upper: Sequence[float],
                     kinematics: CompactionKinematics) -> None:
        """world.rs:1931-2054: the cell shrinks to the new bounds and the
        active fibers follow by `kinematics`; the next batch rebuilds the
        lists on a grid of the same cell size."""
        lower = np.ascontiguousarray(new_lower, dtype=np.float32)
        upper = np.ascontiguousarray(new_upper, dtype=np.float32)
        if lower.size != 3 or upper.size != 3:
            raise ValueError("cell bounds need three coordinates")
        self._fh_compact(lower, upper, int(CompactionKinematics(kinematics)))

    def cell_bounds(self) -> Tuple[List[float], List[float]]:
        """world.rs:2133-2137."""
        lower, upper = self._fh_cell_bounds()
        return [float(v) for v in lower], [float(v) for v in upper]

    def compaction_metrics(self, correction_fraction: float,
                           model: Optional[CompactionEnergyModel] = None) -> CompactionMetrics:
        """world.rs:2056-2117: pressures and penalty energies of the last
        batch's state."""
        model = model or CompactionEnergyModel()
        if not correction_fraction > 0.0:
            raise ValueError("correction_fraction must be positive")
        stiffness = np.array([model.contact_stiffness, model.stretch_stiffness, model.bending_stiffness],
                             dtype=np.float32)
        if np.any(stiffness < 0.0):
            raise ValueError("energy stiffnesses must be non-negative")
        out = self._fh_metrics(float(correction_fraction), stiffness)
        self._last_metrics = out
        return CompactionMetrics((float(out[0]), float(out[1]), float(out[2])), float(out[3]), float(out[4]),
                                 float(out[5]), float(out[6]))

    def wall_face_pressures(self) -> List[List[float]]:
        """world.rs:2119-2131: [lower, upper] pressure on each axis's faces
        from the most recent compaction_metrics call."""
        out = self._last_metrics if self._last_metrics is not None else np.zeros(13, dtype=np.float32)
        return [[float(out[7]), float(out[8])], [float(out[9]), float(out[10])], [float(out[11]), float(out[12])]]

    def wall_reactions(self) -> np.ndarray:
        """The wall reactions of the last update step (interleaved xyz)."""
        return self._fh_wall_reactions()

    # ---- curvature limits

    def set_fiber_maximum_curvatures(self, maximum_curvatures: Sequence[float]) -> None:
        """world.rs:2185-2194: every vertex of fiber f (its ends included)
        takes maximum_curvatures[f] (1 / length; 0 = no limit)."""
        values = np.ascontiguousarray(maximum_curvatures, dtype=np.float32)
        if values.size != self._packed.fiber_count:
            raise ValueError("one curvature limit per fiber")
        self._fh_set_fiber_curvatures(values)
        spans = np.asarray(self._packed.fiber_vertex_spans, dtype=np.int64).reshape(-1, 2)
        self._vertex_max_curvature = np.repeat(values, spans[:, 1])

    @property
    def vertex_max_curvature(self) -> np.ndarray:
        if self._vertex_max_curvature is None:
            return np.asarray(self._packed.vertex_max_curvature, dtype=np.float32).copy()
        return self._vertex_max_curvature.copy()

    # ---- restore

    def _restore_formation(self, checkpoint) -> None:
        """Re-installs the formation state a checkpoint carries."""
        active = np.asarray(checkpoint.packed.fiber_active)
        if not np.all(active):
            self.set_active_fibers(active)
        if checkpoint.wall_reactions is not None:
            self._fh_set_wall_reactions(np.ascontiguousarray(checkpoint.wall_reactions, dtype=np.float32))
        target = checkpoint.layer_target
        if target is not None:
            self._layer_range(target.axis, np.ascontiguousarray(target.coordinates, dtype=np.float32),
                              target.first_layer, target.last_layer, target.stiffness, target.max_translation, False)
        target = checkpoint.vertex_target
        if target is not None:
            self._fh_set_vertex_targets(target.axis, np.ascontiguousarray(target.indices, dtype=np.uint32), 0.0,
                                        target.stiffness, target.max_translation,
                                        np.ascontiguousarray(target.coordinates, dtype=np.float32),
                                        np.ascontiguousarray(target.command_coordinates, dtype=np.float32))
            self._vertex_indices = np.asarray(target.indices, dtype=np.uint32).copy()
            self._vertex_gains = (target.axis, target.stiffness, target.max_translation)
