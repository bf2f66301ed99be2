"""Fiber assemblies and their packed device layout.

`FiberAssembly` is the host data model of a relaxation input: fibers as
polylines with a placed (current) and an intrinsic (rest) shape, a circular
section, and an optional bend limit, inside an orthorhombic cell.
`PackedAssembly` is the flat structure-of-arrays layout the relaxation world
uploads; it follows the reference's non-adaptive packing
(crates/tangle_relax/src/device/packed.rs:150-320):

* positions and intrinsic positions are the f64 points cast to f32,
  interleaved xyz;
* segment i of a fiber joins its vertices i and i+1; the rest length is the
  f64 distance of the intrinsic points, cast to f32 (packed.rs:1058-1063);
* vertex_segments holds (previous, next) segment per vertex, 0xFFFFFFFF at
  the fiber ends;
* vertex_max_curvature is 1/min_bend_radius (f64 reciprocal, cast to f32) on
  interior vertices only, 0 (unrestricted) elsewhere (packed.rs:260-270,
  crates/tangle_core/src/admissibility.rs:10-12);
* pin_fiber_ends pins the first and last vertex of every fiber;
* fiber_formation_steps / fiber_formation_layers carry each fiber's
  formation step (0 by default) and layer (0xFFFFFFFF for none), and
  fiber_active which fibers take part (all of them by default; packed.rs:
  201-210, 289-303).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

NONE = 0xFFFFFFFF


def _parse_periodic(periodic) -> List[bool]:
    if isinstance(periodic, str):
        text = periodic.lower()
        for char in text:
            if char not in "xyz":
                raise ValueError(f"periodic axes must be drawn from 'xyz', got {periodic!r}")
        return ["x" in text, "y" in text, "z" in text]
    values = [bool(v) for v in periodic]
    if len(values) != 3:
        raise ValueError("periodic needs three flags")
    return values


class Cell:
    """Orthorhombic simulation box. `lengths` in metres; `periodic` names the
    periodic axes ("xy", "xyz", ...) or gives three flags. Mirrors
    crates/tangle_python/python/tangle/_tangle.pyi:221-241."""

    def __init__(self, lengths: Sequence[float], periodic="", origin: Sequence[float] = (0.0, 0.0, 0.0)):
        lengths = [float(v) for v in lengths]
        if len(lengths) != 3 or not all(math.isfinite(v) and v > 0.0 for v in lengths):
            raise ValueError("cell lengths must be three positive finite values")
        origin = [float(v) for v in origin]
        if len(origin) != 3 or not all(math.isfinite(v) for v in origin):
            raise ValueError("cell origin must be three finite values")
        self._lengths = lengths
        self._periodic = _parse_periodic(periodic)
        self._origin = origin

    @property
    def lengths(self) -> List[float]:
        return list(self._lengths)

    @property
    def periodic(self) -> List[bool]:
        return list(self._periodic)

    @property
    def origin(self) -> List[float]:
        return list(self._origin)

    def __repr__(self) -> str:
        axes = "".join(a for a, p in zip("xyz", self._periodic) if p)
        return f"Cell(lengths={self._lengths}, periodic={axes!r}, origin={self._origin})"


def py_float(value: float) -> str:
    """A float as the reference's Python reprs print it
    (crates/tangle_python/src/common.rs:250-269): rounded to ten significant
    digits, then Python's own repr (exponent form below 1e-4 and from 1e16,
    with a two-digit exponent; a trailing .0 on whole numbers)."""
    return repr(float(f"{float(value):.9e}"))


class Material:
    """A round fiber type: `diameter` in metres and an optional
    `min_bend_radius` the relaxation keeps fibers above (_tangle.pyi:243-266)."""

    def __init__(self, name: str, diameter: float, min_bend_radius: Optional[float] = None):
        diameter = float(diameter)
        if not (math.isfinite(diameter) and diameter > 0.0):
            raise ValueError("diameter must be positive and finite")
        if min_bend_radius is not None:
            min_bend_radius = float(min_bend_radius)
            if not (math.isfinite(min_bend_radius) and min_bend_radius > 0.0):
                raise ValueError("min_bend_radius must be positive and finite")
        self._name = str(name)
        self._diameter = diameter
        self._min_bend_radius = min_bend_radius

    name = property(lambda self: self._name)
    diameter = property(lambda self: self._diameter)
    radius = property(lambda self: 0.5 * self._diameter)
    min_bend_radius = property(lambda self: self._min_bend_radius)

    def __repr__(self) -> str:
        text = f'Material(name="{self._name}", diameter={py_float(self._diameter)}'
        if self._min_bend_radius is not None:
            text += f", min_bend_radius={py_float(self._min_bend_radius)}"
        return text + ")"


@dataclass
class Fiber:
    placed: np.ndarray  # (n, 3) f64
    intrinsic: np.ndarray  # (n, 3) f64
    radius: float
    min_bend_radius: Optional[float] = None
    formation_step: int = 0  # recipe step that inserts the fiber (assembly.rs formation_step)
    formation_layer: Optional[int] = None  # manufacturing layer (assembly.rs formation_layer)
    material: Optional[str] = None  # material name (assembly.rs materials table)


@dataclass
class FiberAssembly:
    """Fibers placed in a cell (crates/tangle_core/src/assembly.rs:11)."""

    cell: Cell
    fibers: List[Fiber] = field(default_factory=list)

    def add_fiber(self, placed, intrinsic=None, *, radius: float, min_bend_radius: Optional[float] = None,
                  material: Optional[str] = None, formation_layer: Optional[int] = None) -> int:
        placed = np.asarray(placed, dtype=np.float64).reshape(-1, 3)
        intrinsic = placed.copy() if intrinsic is None else np.asarray(intrinsic, dtype=np.float64).reshape(-1, 3)
        if placed.shape[0] < 2:
            raise ValueError("a fiber needs at least two vertices")
        if intrinsic.shape != placed.shape:
            raise ValueError("intrinsic and placed shapes must have the same vertex count")
        if not (np.all(np.isfinite(placed)) and np.all(np.isfinite(intrinsic))):
            raise ValueError("fiber coordinates must be finite")
        if not (math.isfinite(radius) and radius > 0.0):
            raise ValueError("fiber radius must be positive and finite")
        self.fibers.append(Fiber(placed, intrinsic, float(radius), min_bend_radius, 0, None, material))
        if formation_layer is not None:
            self.set_fiber_formation_layer(len(self.fibers) - 1, formation_layer)
        return len(self.fibers) - 1

    @property
    def fiber_count(self) -> int:
        return len(self.fibers)

    def set_fiber_formation_step(self, fiber: int, step: int) -> None:
        """FiberAssembly::set_fiber_formation_step: the recipe step whose
        activation inserts the fiber."""
        step = int(step)
        if not 0 <= step < NONE:
            raise ValueError("formation step must fit in 32 bits")
        self.fibers[fiber].formation_step = step

    def set_fiber_formation_layer(self, fiber: int, layer: Optional[int]) -> None:
        """FiberAssembly::set_fiber_formation_layer: the manufacturing layer
        that layer targets address (None for none)."""
        if layer is not None and not 0 <= int(layer) < NONE:
            raise ValueError("formation layer must fit in 32 bits")
        self.fibers[fiber].formation_layer = None if layer is None else int(layer)

    def smallest_diameter(self) -> Optional[float]:
        if not self.fibers:
            return None
        return min(2.0 * f.radius for f in self.fibers)

    def centerlines(self) -> List[List[List[float]]]:
        return [f.placed.tolist() for f in self.fibers]


@dataclass
class PackedAssembly:
    """Structure-of-arrays device input (packed.rs:49-112, round subset)."""

    positions: np.ndarray  # f32 [3V]
    intrinsic_positions: np.ndarray  # f32 [3V]
    segment_vertices: np.ndarray  # u32 [2S]
    segment_fibers: np.ndarray  # u32 [S]
    segment_radii: np.ndarray  # f32 [S]
    segment_rest_lengths: np.ndarray  # f32 [S]
    fiber_vertex_spans: np.ndarray  # u32 [2F]
    fiber_segment_spans: np.ndarray  # u32 [2F]
    vertex_segments: np.ndarray  # u32 [2V]
    vertex_max_curvature: np.ndarray  # f32 [V]
    vertex_pinned: np.ndarray  # u32 [V]
    cell_lower: np.ndarray  # f32 [3]
    cell_upper: np.ndarray  # f32 [3]
    cell_periodic: np.ndarray  # u32 [3]
    fiber_formation_steps: Optional[np.ndarray] = None  # u32 [F]
    fiber_formation_layers: Optional[np.ndarray] = None  # u32 [F], NONE = no layer
    fiber_active: Optional[np.ndarray] = None  # u32 [F], 1 = takes part

    def __post_init__(self):
        F = self.fiber_vertex_spans.size // 2
        if self.fiber_formation_steps is None:
            self.fiber_formation_steps = np.zeros(F, dtype=np.uint32)
        if self.fiber_formation_layers is None:
            self.fiber_formation_layers = np.full(F, NONE, dtype=np.uint32)
        if self.fiber_active is None:
            self.fiber_active = np.ones(F, dtype=np.uint32)

    @property
    def vertex_count(self) -> int:
        return self.positions.size // 3

    @property
    def segment_count(self) -> int:
        return self.segment_fibers.size

    @property
    def fiber_count(self) -> int:
        return self.fiber_vertex_spans.size // 2

    @staticmethod
    def from_assembly(assembly: FiberAssembly, pin_fiber_ends: bool = False) -> "PackedAssembly":
        """packed.rs:150-320 for round, non-adaptive fibers."""
        if not assembly.fibers:
            raise ValueError("assembly has no fibers")
        counts = np.array([f.placed.shape[0] for f in assembly.fibers], dtype=np.int64)
        V = int(counts.sum())
        S = int((counts - 1).sum())
        F = len(assembly.fibers)
        if V >= NONE or S >= NONE:
            raise ValueError("assembly too large for 32-bit indices")
        vstart = np.zeros(F, dtype=np.int64)
        vstart[1:] = np.cumsum(counts)[:-1]
        sstart = vstart - np.arange(F, dtype=np.int64)
        placed = np.concatenate([f.placed for f in assembly.fibers], axis=0)
        intrinsic = np.concatenate([f.intrinsic for f in assembly.fibers], axis=0)
        positions = placed.astype(np.float32).reshape(-1)
        intrinsic_positions = intrinsic.astype(np.float32).reshape(-1)

        fiber_of_vertex = np.repeat(np.arange(F, dtype=np.int64), counts)
        local = np.arange(V, dtype=np.int64) - vstart[fiber_of_vertex]
        is_last = local == counts[fiber_of_vertex] - 1
        seg_first = np.nonzero(~is_last)[0]  # first vertex of every segment, in order
        segment_vertices = np.stack([seg_first, seg_first + 1], axis=1).astype(np.uint32).reshape(-1)
        segment_fibers = fiber_of_vertex[seg_first].astype(np.uint32)
        radii = np.array([np.float32(f.radius) for f in assembly.fibers], dtype=np.float32)
        segment_radii = radii[segment_fibers]
        delta = intrinsic[seg_first + 1] - intrinsic[seg_first]
        segment_rest_lengths = np.sqrt(
            delta[:, 0] * delta[:, 0] + delta[:, 1] * delta[:, 1] + delta[:, 2] * delta[:, 2]
        ).astype(np.float32)

        fiber_vertex_spans = np.stack([vstart, counts], axis=1).astype(np.uint32).reshape(-1)
        fiber_segment_spans = np.stack([sstart, counts - 1], axis=1).astype(np.uint32).reshape(-1)

        vertex_segments = np.full((V, 2), NONE, dtype=np.uint32)
        seg_index = np.arange(S, dtype=np.uint32)
        vertex_segments[seg_first, 1] = seg_index
        vertex_segments[seg_first + 1, 0] = seg_index

        vertex_max_curvature = np.zeros(V, dtype=np.float32)
        interior = (local > 0) & ~is_last
        limits = np.array(
            [0.0 if f.min_bend_radius is None else float(np.float32(1.0 / f.min_bend_radius)) for f in assembly.fibers],
            dtype=np.float32,
        )
        vertex_max_curvature[interior] = limits[fiber_of_vertex[interior]]

        vertex_pinned = np.zeros(V, dtype=np.uint32)
        if pin_fiber_ends:
            vertex_pinned[vstart] = 1
            vertex_pinned[vstart + counts - 1] = 1

        cell = assembly.cell
        lower = np.array(cell.origin, dtype=np.float64)
        upper = lower + np.array(cell.lengths, dtype=np.float64)
        return PackedAssembly(
            positions=positions,
            intrinsic_positions=intrinsic_positions,
            segment_vertices=segment_vertices,
            segment_fibers=segment_fibers,
            segment_radii=segment_radii,
            segment_rest_lengths=segment_rest_lengths,
            fiber_vertex_spans=fiber_vertex_spans,
            fiber_segment_spans=fiber_segment_spans,
            vertex_segments=vertex_segments.reshape(-1),
            vertex_max_curvature=vertex_max_curvature,
            vertex_pinned=vertex_pinned,
            cell_lower=lower.astype(np.float32),
            cell_upper=upper.astype(np.float32),
            cell_periodic=np.array([1 if p else 0 for p in cell.periodic], dtype=np.uint32),
            fiber_formation_steps=np.array([f.formation_step for f in assembly.fibers], dtype=np.uint32),
            fiber_formation_layers=np.array(
                [NONE if f.formation_layer is None else f.formation_layer for f in assembly.fibers], dtype=np.uint32),
        )

    def unpack_positions(self, positions: np.ndarray, assembly: FiberAssembly) -> None:
        """Installs downloaded f32 positions as the placed f64 points
        (packed.rs unpack_positions for a non-adaptive layout)."""
        positions = np.asarray(positions, dtype=np.float32).reshape(-1, 3).astype(np.float64)
        spans = self.fiber_vertex_spans.reshape(-1, 2)
        for fiber, (start, count) in zip(assembly.fibers, spans):
            fiber.placed = positions[start : start + count].copy()
