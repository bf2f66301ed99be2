"""Solver settings: the reference's RelaxationConfig / CellListConfig /
BatchStatus and the Python-facing RelaxationSettings.

* `CellListConfig` -- crates/tangle_contact/src/lib.rs:15-40 (defaults 1.0,
  2.0, 48) plus `max_list_bytes`, the neighbor-list buffer cap. The reference
  fixes the cap at 120 MiB for WGPU binding limits
  (crates/tangle_relax/src/device/world.rs:35-36); 0 keeps that value.
  The cap only decides which segments take the exact cell-scan fallback,
  never which contacts are found.
* `RelaxationConfig` -- crates/tangle_relax/src/device/plugin.rs:77-175,
  values rounded to f32 as the solver sees them.
* `BatchStatus` -- crates/tangle_relax/src/device/world.rs:91-114.
* `RelaxationSettings` -- crates/tangle_python/src/settings.rs:474-609 and
  crates/tangle_python/python/tangle/_tangle.pyi:712-779: same field names,
  defaults, validation messages and diameter-scaled defaults
  (`penetration_tolerance` = 1 % and `max_step` = 10 % of the smallest fiber
  diameter when unset, settings.rs:474).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field, fields, replace
from typing import Optional

import numpy as np

#: settings.rs:474 -- unset lengths as fractions of the smallest diameter.
DIAMETER_FRACTIONS = (0.01, 0.1)
REFERENCE_MAX_LIST_BYTES = 120 << 20

_AGGREGATIONS = {"uniform_average": 0, "penetration_weighted": 1, "deepest_only": 2}
_MOTION_MODELS = ("flexible", "rigid_translation")
#: Backends of the reference's seam (settings.rs:16-21). This build provides
#: "cuda" only; the others belong to the reference.
_BACKENDS = ("wgpu", "cpu", "cuda")


def f32(value: float) -> float:
    return float(np.float32(value))


@dataclass
class CellListConfig:
    cell_size_scale: float = 1.0
    neighbor_skin_scale: float = 2.0
    neighbor_capacity: int = 48
    max_list_bytes: int = 0


@dataclass
class RelaxationConfig:
    penetration_tolerance: float = 1.0e-4
    force_full_iterations: bool = False
    correction_fraction: float = 0.8
    contact_aggregation: int = 0
    stretch_stiffness: float = 0.35
    bend_stiffness: float = 0.03
    curvature_limit_stiffness: float = 1.0
    curvature_limit_safety_margin: float = 1.0e-3
    curvature_ratio_tolerance: float = 1.0e-5
    constraint_iterations: int = 2
    curvature_cleanup_sweeps: int = 4
    max_step: float = 0.006
    max_iterations: int = 2000
    iterations_per_batch: int = 128
    pin_fiber_ends: bool = False
    motion_model: str = "flexible"
    cell_list: CellListConfig = field(default_factory=CellListConfig)

    def validate(self) -> None:
        """plugin.rs:951-983 assertions, raised as ValueError."""
        checks = [
            (self.penetration_tolerance >= 0.0, "penetration_tolerance must be non-negative"),
            (0.0 < self.correction_fraction <= 1.0, "correction_fraction must be in (0, 1]"),
            (0.0 <= self.stretch_stiffness <= 1.0, "stretch_stiffness must be in [0, 1]"),
            (0.0 <= self.bend_stiffness <= 1.0, "bend_stiffness must be in [0, 1]"),
            (0.0 <= self.curvature_limit_stiffness <= 1.0, "curvature_limit_stiffness must be in [0, 1]"),
            (0.0 <= self.curvature_limit_safety_margin < 0.1, "curvature_limit_safety_margin must be in [0, 0.1)"),
            (self.curvature_ratio_tolerance >= 0.0, "curvature_ratio_tolerance must be non-negative"),
            (self.constraint_iterations > 0, "constraint_iterations must be positive"),
            (self.curvature_cleanup_sweeps > 0, "curvature_cleanup_sweeps must be positive"),
            (self.max_step > 0.0, "max_step must be positive"),
            (self.max_iterations > 0, "max_iterations must be positive"),
            (self.iterations_per_batch > 0, "iterations_per_batch must be positive"),
            (self.cell_list.cell_size_scale >= 1.0, "cell_size_scale must be at least 1"),
            (self.contact_aggregation in (0, 1, 2), "contact_aggregation must be 0, 1 or 2"),
        ]
        for ok, message in checks:
            if not ok:
                raise ValueError(message)
        if self.motion_model not in _MOTION_MODELS:
            raise ValueError(f"motion_model must be one of {', '.join(_MOTION_MODELS)}")

    @property
    def motion_code(self) -> int:
        """FiberMotion as the C ABI's motion_model: 0 flexible, 1 rigid translation."""
        return _MOTION_MODELS.index(self.motion_model)


@dataclass
class BatchStatus:
    total_iterations: int = 0
    batch_iterations: int = 0
    max_penetration: float = 0.0
    max_displacement: float = 0.0
    max_curvature_ratio: float = 0.0
    converged: bool = False
    cell_list_overflow: bool = False


def _check_unit(name: str, value: float) -> None:
    if not math.isfinite(value) or not (0.0 <= value <= 1.0) or (value == 0.0 and name == "correction_fraction"):
        raise ValueError(f"{name} must be finite and within its [0, 1] range")


@dataclass
class RelaxationSettings:
    """Run-wide solver settings for `Recipe.run` (_tangle.pyi:712-779).

    `backend` names the relaxation seam's implementation. This library is the
    "cuda" implementation; "wgpu" and "cpu" are the reference's own backends
    and are rejected by `to_config` here. Unset, `penetration_tolerance` is
    1 % and `max_step` 10 % of the smallest fiber diameter in the recipe.
    """

    backend: str = "cuda"
    motion_model: str = "flexible"
    pin_fiber_ends: bool = False
    penetration_tolerance: Optional[float] = None
    force_full_iterations: bool = False
    correction_fraction: float = 0.8
    contact_aggregation: str = "uniform_average"
    stretch_stiffness: float = 0.35
    bend_stiffness: float = 0.03
    curvature_limit_stiffness: float = 1.0
    curvature_limit_safety_margin: float = 1.0e-3
    curvature_ratio_tolerance: float = 1.0e-5
    constraint_iterations: int = 2
    curvature_cleanup_sweeps: int = 4
    twist_stiffness: float = 0.1
    keep_rest_twist: bool = False
    junction_stiffness: float = 0.0
    max_step: Optional[float] = None
    max_iterations: int = 2000
    iterations_per_batch: int = 128
    debug_snapshot_interval: Optional[int] = None
    save_assembled_reference: bool = True
    cell_size_scale: float = 1.0
    neighbor_skin_scale: float = 2.0
    neighbor_capacity: int = 48
    max_list_bytes: int = 0
    adaptive_segmentation: Optional[object] = None

    def __post_init__(self):
        if self.backend not in _BACKENDS:
            raise ValueError(f"backend must be one of {', '.join(_BACKENDS)}")
        if self.motion_model not in _MOTION_MODELS:
            raise ValueError(f"motion_model must be one of {', '.join(_MOTION_MODELS)}")
        if self.contact_aggregation not in _AGGREGATIONS:
            raise ValueError(f"contact_aggregation must be one of {', '.join(_AGGREGATIONS)}")

    def copy(self) -> "RelaxationSettings":
        return replace(self)

    def replace(self, **changes) -> "RelaxationSettings":
        names = {f.name for f in fields(self)}
        for key in changes:
            if key not in names:
                raise TypeError(f"unknown RelaxationSettings field {key!r}")
        return replace(self, **changes)

    def to_dict(self) -> dict:
        return {f.name: getattr(self, f.name) for f in fields(self)}

    def to_config(self, smallest_diameter: Optional[float] = None) -> RelaxationConfig:
        """settings.rs:485-609 (`to_rust_for`)."""
        tolerance_fraction, step_fraction = DIAMETER_FRACTIONS
        defaults = RelaxationConfig()
        if self.penetration_tolerance is not None:
            penetration_tolerance = float(self.penetration_tolerance)
        elif smallest_diameter is not None:
            penetration_tolerance = tolerance_fraction * smallest_diameter
        else:
            penetration_tolerance = defaults.penetration_tolerance
        if self.max_step is not None:
            max_step = float(self.max_step)
        elif smallest_diameter is not None:
            max_step = step_fraction * smallest_diameter
        else:
            max_step = defaults.max_step
        if not math.isfinite(penetration_tolerance) or penetration_tolerance < 0.0:
            raise ValueError("penetration_tolerance must be nonnegative and finite")
        for name in ("correction_fraction", "stretch_stiffness", "bend_stiffness", "curvature_limit_stiffness",
                     "twist_stiffness", "junction_stiffness"):
            _check_unit(name, float(getattr(self, name)))
        if not math.isfinite(self.curvature_limit_safety_margin) or not (0.0 <= self.curvature_limit_safety_margin < 0.1):
            raise ValueError("curvature_limit_safety_margin must be in [0, 0.1)")
        if not math.isfinite(self.curvature_ratio_tolerance) or self.curvature_ratio_tolerance < 0.0:
            raise ValueError("curvature_ratio_tolerance must be nonnegative and finite")
        if (self.constraint_iterations == 0 or self.curvature_cleanup_sweeps == 0 or self.max_iterations == 0
                or self.iterations_per_batch == 0):
            raise ValueError("iteration and sweep counts must be positive")
        if not math.isfinite(max_step) or max_step <= 0.0:
            raise ValueError("max_step must be positive and finite")
        if not math.isfinite(self.cell_size_scale) or self.cell_size_scale < 1.0:
            raise ValueError("cell_size_scale must be finite and at least 1")
        if not math.isfinite(self.neighbor_skin_scale) or self.neighbor_skin_scale < 0.0:
            raise ValueError("neighbor_skin_scale must be finite and non-negative")
        if self.neighbor_capacity == 0:
            raise ValueError("neighbor_capacity must be at least 1")
        if self.debug_snapshot_interval == 0:
            raise ValueError("debug_snapshot_interval must be positive when supplied")
        if self.adaptive_segmentation is not None:
            raise ValueError("adaptive segmentation is not provided by the CUDA relaxation path")
        if self.junction_stiffness != 0.0:
            raise ValueError("junction tethers are not provided by the CUDA relaxation path")
        config = RelaxationConfig(
            penetration_tolerance=f32(penetration_tolerance),
            force_full_iterations=bool(self.force_full_iterations),
            correction_fraction=f32(self.correction_fraction),
            contact_aggregation=_AGGREGATIONS[self.contact_aggregation],
            stretch_stiffness=f32(self.stretch_stiffness),
            bend_stiffness=f32(self.bend_stiffness),
            curvature_limit_stiffness=f32(self.curvature_limit_stiffness),
            curvature_limit_safety_margin=f32(self.curvature_limit_safety_margin),
            curvature_ratio_tolerance=f32(self.curvature_ratio_tolerance),
            constraint_iterations=int(self.constraint_iterations),
            curvature_cleanup_sweeps=int(self.curvature_cleanup_sweeps),
            max_step=f32(max_step),
            max_iterations=int(self.max_iterations),
            iterations_per_batch=int(self.iterations_per_batch),
            pin_fiber_ends=bool(self.pin_fiber_ends),
            motion_model=self.motion_model,
            cell_list=CellListConfig(
                cell_size_scale=f32(self.cell_size_scale),
                neighbor_skin_scale=f32(self.neighbor_skin_scale),
                neighbor_capacity=int(self.neighbor_capacity),
                max_list_bytes=int(self.max_list_bytes),
            ),
        )
        config.validate()
        return config
