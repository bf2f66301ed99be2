"""Needling: which vertices a needle pulls (crates/tangle_generate/src/
recipe.rs:233-300, :1688-1812; Python classes crates/tangle_python/src/
recipe.rs:64-140).

A needle command pulls at most one internal vertex of each chosen fiber of
one formation layer toward the negative layer-normal direction, through the
world's vertex displacement targets. The fibers are chosen by a footprint:

* `RandomFiberFraction(fraction, seed=0)` -- each layer fiber independently
  with probability `fraction` (a SplitMix64 draw seeded by seed ^ fiber id),
  pulling one of its internal vertices drawn the same way;
* `CircularFootprint(center, diameter=...)` -- every layer fiber whose
  centerline crosses a circle in the layer plane (minimum image on periodic
  plane axes), pulling its vertex nearest the circle's centre;
  `CircularFootprint.random(diameter=..., seed=...)` places the centre
  reproducibly per layer, uniform over the cell's footprint.

All geometry is in f32, in the reference's order of operations. A fiber's id
is its index in the assembly plus one.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

MASK64 = (1 << 64) - 1


def splitmix64(value: int) -> int:
    """One SplitMix64 output for state `value` (recipe.rs:1814-1819)."""
    value = (value + 0x9E3779B97F4A7C15) & MASK64
    value = ((value ^ (value >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    value = ((value ^ (value >> 27)) * 0x94D049BB133111EB) & MASK64
    return value ^ (value >> 31)


def random_footprint_center(seed: int, layer: int, origin: Sequence[float], extent: Sequence[float]) -> List[float]:
    """recipe.rs:233-246: a reproducible centre per layer, uniform over the
    footprint (24-bit units, f32)."""
    f32 = np.float32

    def unit(bits: int):
        return f32(float(bits >> 40) * (1.0 / float(1 << 24)))

    first = splitmix64((seed ^ (2 * layer)) & MASK64)
    second = splitmix64((seed ^ (2 * layer + 1)) & MASK64)
    return [float(f32(origin[0]) + f32(extent[0]) * unit(first)),
            float(f32(origin[1]) + f32(extent[1]) * unit(second))]


@dataclass(frozen=True)
class CircularFootprint:
    """Pull fibers whose centerline crosses a circle in the layer plane."""

    center: Optional[Sequence[float]]
    diameter: float
    seed: Optional[int] = None

    def __init__(self, center: Sequence[float], *, diameter: float):
        if len(center) != 2 or not all(math.isfinite(float(v)) for v in center):
            raise ValueError("footprint center must be finite")
        if not (math.isfinite(float(diameter)) and float(diameter) > 0.0):
            raise ValueError("diameter must be positive and finite")
        object.__setattr__(self, "center", [float(v) for v in center])
        object.__setattr__(self, "diameter", float(diameter))
        object.__setattr__(self, "seed", None)

    @classmethod
    def random(cls, *, diameter: float, seed: int) -> "CircularFootprint":
        if not (math.isfinite(float(diameter)) and float(diameter) > 0.0):
            raise ValueError("diameter must be positive and finite")
        footprint = cls.__new__(cls)
        object.__setattr__(footprint, "center", None)
        object.__setattr__(footprint, "diameter", float(diameter))
        object.__setattr__(footprint, "seed", int(seed))
        return footprint


@dataclass(frozen=True)
class RandomFiberFraction:
    """Pull a seeded random `fraction` of the layer's fibers."""

    fraction: float
    seed: int = 0

    def __post_init__(self):
        if not (0.0 < float(self.fraction) <= 1.0):
            raise ValueError("fraction must be in (0, 1]")


@dataclass
class NeedlingConfig:
    """recipe.rs:268-286."""

    layer: int
    footprint: object  # RandomFiberFraction or CircularFootprint with a centre
    depth: float
    stiffness: float = 0.25
    max_translation: float = 1.0e-5
    max_translation_over_diameter: float = 0.25
    min_fiber_diameter: Optional[float] = None


def selected_needling_vertices(assembly, packed, positions: np.ndarray, fiber_active: np.ndarray,
                               active_through: Optional[int], layer_axis: int, config: NeedlingConfig) -> List[int]:
    """recipe.rs:1710-1812: at most one internal vertex per selected fiber of
    `config.layer` that is active and was inserted through `active_through`,
    in fiber order."""
    f32 = np.float32
    plane = [a for a in range(3) if a != layer_axis]
    xyz = np.asarray(positions, dtype=np.float32).reshape(-1)
    vspans = np.asarray(packed.fiber_vertex_spans).reshape(-1, 2)
    sspans = np.asarray(packed.fiber_segment_spans).reshape(-1, 2)
    seg_vertices = np.asarray(packed.segment_vertices).reshape(-1, 2)
    out = []
    for index, fiber in enumerate(assembly.fibers):
        if fiber.formation_layer != config.layer:
            continue
        if active_through is not None and fiber.formation_step > active_through:
            continue
        if config.min_fiber_diameter is not None and 2.0 * fiber.radius < float(f32(config.min_fiber_diameter)):
            continue
        start, count = int(vspans[index, 0]), int(vspans[index, 1])
        active = [v for v in range(start, start + count) if fiber_active[index]]
        footprint = config.footprint
        if isinstance(footprint, RandomFiberFraction):
            if len(active) <= 2:
                continue
            selection = splitmix64(int(footprint.seed) ^ (index + 1))
            unit = float(selection >> 11) * (1.0 / float(1 << 53))
            if unit >= float(f32(footprint.fraction)):
                continue
            internal = len(active) - 2
            out.append(active[1 + splitmix64(selection) % internal])
            continue
        center = [f32(v) for v in footprint.center]
        diameter = f32(footprint.diameter)
        if not fiber_active[index]:
            continue
        best = None
        s0, m = int(sspans[index, 0]), int(sspans[index, 1])
        for segment in range(s0, s0 + m):
            first, second = int(seg_vertices[segment, 0]), int(seg_vertices[segment, 1])
            start_delta, direction = [f32(0.0), f32(0.0)], [f32(0.0), f32(0.0)]
            for k, axis in enumerate(plane):
                start_delta[k] = xyz[3 * first + axis] - center[k]
                direction[k] = xyz[3 * second + axis] - xyz[3 * first + axis]
                if packed.cell_periodic[axis]:
                    width = f32(packed.cell_upper[axis]) - f32(packed.cell_lower[axis])
                    start_delta[k] = start_delta[k] - f32(_round_half_away(start_delta[k] / width)) * width
                    direction[k] = direction[k] - f32(_round_half_away(direction[k] / width)) * width
            length_squared = direction[0] * direction[0] + direction[1] * direction[1]
            if length_squared > f32(1.0e-20):
                coordinate = -(start_delta[0] * direction[0] + start_delta[1] * direction[1]) / length_squared
                coordinate = min(max(coordinate, f32(0.0)), f32(1.0))
            else:
                coordinate = f32(0.0)
            dx = start_delta[0] + coordinate * direction[0]
            dy = start_delta[1] + coordinate * direction[1]
            radius_squared = dx * dx + dy * dy
            if radius_squared > f32(0.25) * diameter * diameter:
                continue
            material = _round_half_away(f32(first) + coordinate * f32(second - first))
            vertex = min(max(int(material), start + 1), start + count - 2)
            if best is None or radius_squared < best[1]:
                best = (vertex, radius_squared)
        if best is not None:
            out.append(best[0])
    return out


def _round_half_away(x) -> float:
    """Rust f32::round: half-way cases away from zero."""
    x = float(x)
    return math.floor(x + 0.5) if x >= 0.0 else -math.floor(-x + 0.5)
