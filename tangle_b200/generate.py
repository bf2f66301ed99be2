"""Seeded synthetic fiber inputs.

* `SplitMix64` -- the reference's generator, bit for bit
  (crates/tangle_generate/src/population.rs:795-812): 53-bit unit doubles.
* `FiberPopulation` / `generate_fiber_population` -- the reference's biased
  box generator (population.rs:246-357) for isotropic orientation and uniform
  position: per fiber it draws length, radius, waviness amplitude and
  handedness, builds the local centerline (population.rs:554-565), draws a
  direction (population.rs:567-578) and a contained centre
  (population.rs:657-693), in that order. Python defaults follow
  crates/tangle_python/src/generators.rs:395-450 (length 16-24 diameters,
  curvature amplitude 0-0.8 diameters, 8 segments, seed 1).
* `mid_size_specimen`, `cpu_runnable_specimen`, `batched_specimens`,
  `ply_stack_specimen` -- the benchmark workloads: synthetic stand-ins with the shapes, sizes and value
  distributions of the configurations they are named after (no dataset is
  involved; every input is generated here from a seed).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, replace
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from .assembly import Cell, FiberAssembly, Material

MASK64 = (1 << 64) - 1


class SplitMix64:
    """population.rs:795-812."""

    def __init__(self, seed: int):
        self.state = int(seed) & MASK64

    def unit(self) -> float:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        value = self.state
        value = ((value ^ (value >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        value = ((value ^ (value >> 27)) * 0x94D049BB133111EB) & MASK64
        value ^= value >> 31
        return float(value >> 11) * (1.0 / float(1 << 53))


def _normalize(v):
    n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return [v[0] / n, v[1] / n, v[2] / n]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def perpendicular(direction):
    """population.rs:758-768."""
    ax, ay, az = abs(direction[0]), abs(direction[1]), abs(direction[2])
    if ax <= ay and ax <= az:
        axis = [1.0, 0.0, 0.0]
    elif ay <= az:
        axis = [0.0, 1.0, 0.0]
    else:
        axis = [0.0, 0.0, 1.0]
    return _normalize(_cross(direction, axis))


def isotropic_direction(random: SplitMix64):
    """population.rs:573-578."""
    z = 2.0 * random.unit() - 1.0
    azimuth = 2.0 * math.pi * random.unit()
    radial = math.sqrt(1.0 - z * z)
    return [radial * math.cos(azimuth), radial * math.sin(azimuth), z]


def schladitz_axis_cosine_quantile(beta: float, p: float) -> float:
    """|cos theta| quantile of the Schladitz orientation density about an
    axis (crates/tangle_characterize/src/shape.rs:550-556)."""
    beta2 = beta * beta
    p = min(max(p, 0.0), 1.0)
    return min(p / math.sqrt(beta2 - (beta2 - 1.0) * p * p), 1.0)


def local_centerline(segments: int, length: float, amplitude: float, handedness: float) -> np.ndarray:
    """population.rs:554-565."""
    points = []
    for index in range(segments + 1):
        centered = index / segments - 0.5
        points.append([
            centered * length,
            amplitude * math.sin(2.0 * math.pi * centered),
            0.5 * amplitude * handedness * math.sin(4.0 * math.pi * centered),
        ])
    return np.array(points, dtype=np.float64)


Range = Union[float, Tuple[float, float], None]


def _range(value: Range) -> Optional[Tuple[float, float]]:
    if value is None:
        return None
    if isinstance(value, (int, float)):
        return (float(value), float(value))
    low, high = value
    return (float(low), float(high))


@dataclass
class FiberPopulation:
    """Random fibers for `generate_fiber_population` (_tangle.pyi:459-500)."""

    material: Material = None
    count: int = 32
    segments_per_fiber: int = 8
    seed: int = 1
    length: Range = None
    diameter: Range = None
    curvature_amplitude: Range = None
    max_attempts_per_fiber: int = 1000

    def __post_init__(self):
        if self.material is None:
            self.material = Material("fiber", 0.025, 0.08)
        if self.count < 0:
            raise ValueError("count must be non-negative")
        if self.segments_per_fiber < 2:
            raise ValueError("segments_per_fiber must be at least 2")

    def copy(self) -> "FiberPopulation":
        return replace(self)

    def replace(self, **changes) -> "FiberPopulation":
        return replace(self, **changes)


def generate_fiber_population(cell: Cell, population: FiberPopulation) -> FiberAssembly:
    """population.rs:246-357, isotropic directions and uniform centres."""
    assembly = FiberAssembly(cell)
    d = population.material.diameter
    length = _range(population.length) or (16.0 * d, 24.0 * d)
    diameter = _range(population.diameter) or (d, d)
    amplitude = _range(population.curvature_amplitude) or (0.0, 0.8 * d)
    min_bend = population.material.min_bend_radius
    random = SplitMix64(population.seed)
    low = np.array(cell.origin)
    high = low + np.array(cell.lengths)
    periodic = cell.periodic
    for fiber_index in range(population.count):
        placed_fiber = None
        for _ in range(population.max_attempts_per_fiber):
            fiber_length = length[0] + (length[1] - length[0]) * random.unit()
            radius = 0.5 * (diameter[0] + (diameter[1] - diameter[0]) * random.unit())
            wave = amplitude[0] + (amplitude[1] - amplitude[0]) * random.unit()
            handedness = -1.0 if random.unit() < 0.5 else 1.0
            intrinsic = local_centerline(population.segments_per_fiber, fiber_length, wave, handedness)
            if min_bend is not None and maximum_polyline_curvature(intrinsic) > (1.0 / min_bend) * (1.0 + 1.0e-10):
                continue
            direction = isotropic_direction(random)
            ta = perpendicular(direction)
            tb = _normalize(_cross(direction, ta))
            offsets = (np.outer(intrinsic[:, 0], direction) + np.outer(intrinsic[:, 1], ta)
                       + np.outer(intrinsic[:, 2], tb))
            lower = np.empty(3)
            upper = np.empty(3)
            ok = True
            for axis in range(3):
                if periodic[axis]:
                    lower[axis], upper[axis] = low[axis], high[axis]
                    continue
                lower[axis] = low[axis] + radius - offsets[:, axis].min()
                upper[axis] = high[axis] - radius - offsets[:, axis].max()
                if lower[axis] > upper[axis]:
                    ok = False
                    break
            if not ok:
                continue
            center = np.array([lower[a] + (upper[a] - lower[a]) * random.unit() for a in range(3)])
            placed_fiber = (intrinsic, center + offsets, radius)
            break
        if placed_fiber is None:
            raise RuntimeError(f"could not place fiber {fiber_index} inside the cell")
        intrinsic, placed, radius = placed_fiber
        assembly.add_fiber(placed, intrinsic, radius=radius, min_bend_radius=min_bend,
                           material=population.material.name)
    return assembly


def sample_orientation(orientation, random: SplitMix64):
    """sample_orientation (crates/tangle_generate/src/population.rs:567-655)
    for the distributions the regression cases use: ("isotropic",),
    ("aligned", axis, maximum_angle) -- a uniform cosine on the cap within
    `maximum_angle` of `axis` and a uniform azimuth -- and ("planar", normal,
    maximum_tilt) -- a uniform in-plane azimuth and a uniform tilt out of the
    plane normal to `normal`."""
    kind = orientation[0]
    if kind == "isotropic":
        return isotropic_direction(random)
    if kind == "aligned":
        axis = _normalize(orientation[1])
        ta = perpendicular(axis)
        tb = _normalize(_cross(axis, ta))
        minimum_cosine = math.cos(orientation[2])
        cosine = minimum_cosine + (1.0 - minimum_cosine) * random.unit()
        sine = math.sqrt(max(1.0 - cosine * cosine, 0.0))
        azimuth = 2.0 * math.pi * random.unit()
        return [axis[i] * cosine + (ta[i] * math.cos(azimuth) + tb[i] * math.sin(azimuth)) * sine for i in range(3)]
    if kind == "planar":
        normal = _normalize(orientation[1])
        a = perpendicular(normal)
        b = _normalize(_cross(normal, a))
        azimuth = 2.0 * math.pi * random.unit()
        tilt = orientation[2] * (2.0 * random.unit() - 1.0)
        return [(a[i] * math.cos(azimuth) + b[i] * math.sin(azimuth)) * math.cos(tilt) + normal[i] * math.sin(tilt)
                for i in range(3)]
    raise ValueError(f"unknown orientation distribution {kind!r}")


def biased_fiber_population(cell: Cell, count: int, segments_per_fiber: int, seed: int, length: Range,
                            radius: Range, curvature_amplitude: Range, orientation=("isotropic",),
                            min_bend_radius: Optional[float] = None, max_attempts_per_fiber: int = 256,
                            material: str = "fiber") -> FiberAssembly:
    """generate_biased_fiber_population (crates/tangle_generate/src/population.rs:
    246-357) with uniform positions: per fiber, draw length, radius, waviness
    and handedness, reject shapes over the bend limit, orient the local
    centerline by `sample_orientation`, and place its centre uniformly where
    the whole fiber (with its radius) lies inside the walls
    (sample_contained_center, :657-700). Ranges are (minimum, maximum)
    uniform draws; a single number is a constant and draws nothing
    (ScalarDistribution::sample, :27-32)."""
    def sample(value, random):
        if isinstance(value, (int, float)):
            return float(value)
        return float(value[0]) + (float(value[1]) - float(value[0])) * random.unit()

    assembly = FiberAssembly(cell)
    random = SplitMix64(seed)
    low = np.array(cell.origin, dtype=np.float64)
    high = low + np.array(cell.lengths, dtype=np.float64)
    for fiber_index in range(count):
        placed_fiber = None
        for _ in range(max_attempts_per_fiber):
            fiber_length = sample(length, random)
            fiber_radius = sample(radius, random)
            wave = sample(curvature_amplitude, random)
            handedness = -1.0 if random.unit() < 0.5 else 1.0
            intrinsic = local_centerline(segments_per_fiber, fiber_length, wave, handedness)
            if min_bend_radius is not None and maximum_polyline_curvature(intrinsic) > (
                    1.0 / min_bend_radius) * (1.0 + 1.0e-10):
                continue
            direction = sample_orientation(orientation, random)
            ta = perpendicular(direction)
            tb = _normalize(_cross(direction, ta))
            offsets = (np.outer(intrinsic[:, 0], direction) + np.outer(intrinsic[:, 1], ta)
                       + np.outer(intrinsic[:, 2], tb))
            lower, upper = low.copy(), high.copy()
            ok = True
            for axis in range(3):
                if cell.periodic[axis]:
                    continue
                lower[axis] = low[axis] + fiber_radius - offsets[:, axis].min()
                upper[axis] = high[axis] - fiber_radius - offsets[:, axis].max()
                if lower[axis] > upper[axis]:
                    ok = False
                    break
            if not ok:
                continue
            center = np.array([lower[a] + (upper[a] - lower[a]) * random.unit() for a in range(3)])
            placed_fiber = (intrinsic, center + offsets, fiber_radius)
            break
        if placed_fiber is None:
            raise RuntimeError(f"could not place fiber {fiber_index} inside the cell")
        intrinsic, placed, fiber_radius = placed_fiber
        assembly.add_fiber(placed, intrinsic, radius=fiber_radius, min_bend_radius=min_bend_radius,
                           material=material)
    return assembly


def orientation_tensor(centerlines) -> np.ndarray:
    """The length-weighted orientation tensor of characterize_assembly
    (crates/tangle_characterize/src/lib.rs:186-300, :447-463): sum over
    segments of length * t t^T, divided by the total length (f64)."""
    tensor = np.zeros((3, 3), dtype=np.float64)
    total = 0.0
    for line in centerlines:
        points = np.asarray(line, dtype=np.float64)
        delta = points[1:] - points[:-1]
        lengths = np.sqrt((delta * delta).sum(axis=1))
        keep = lengths > np.finfo(np.float64).eps
        tangents = delta[keep] / lengths[keep, None]
        tensor += np.einsum("n,ni,nj->ij", lengths[keep], tangents, tangents)
        total += float(lengths[keep].sum())
    return tensor / total if total > np.finfo(np.float64).eps else tensor


def maximum_polyline_curvature(points: np.ndarray) -> float:
    """crates/tangle_core/src/curvature.rs:21-61 (f64)."""
    best = 0.0
    for i in range(1, len(points) - 1):
        a = points[i] - points[i - 1]
        b = points[i + 1] - points[i]
        la, lb = float(np.linalg.norm(a)), float(np.linalg.norm(b))
        if la <= 2.220446049250313e-16 or lb <= 2.220446049250313e-16:
            continue
        cosine = min(max(float(a @ b) / (la * lb), -1.0), 1.0)
        angle = math.acos(cosine)
        curvature = 2.0 * math.sin(0.5 * angle) / (0.5 * (la + lb))
        best = max(best, curvature)
    return best


def _straight_fibers(assembly: FiberAssembly, starts: np.ndarray, directions: np.ndarray, length: float,
                     segments: int, radius: float, min_bend_radius: Optional[float]) -> None:
    steps = np.arange(segments + 1, dtype=np.float64) * (length / segments)
    for start, direction in zip(starts, directions):
        points = start[None, :] + steps[:, None] * direction[None, :]
        assembly.add_fiber(points, points, radius=radius, min_bend_radius=min_bend_radius)


def cpu_runnable_specimen(seed: int = 1) -> FiberAssembly:
    """Periodic 300 um cube, 40 straight 10 um fibers, 300 um long as 30
    segments (31 nodes); first node uniform in the cell, direction uniform on
    the sphere; curvature limit 1/(5 d). 1,240 nodes."""
    d = 10.0e-6
    side = 300.0e-6
    cell = Cell([side] * 3, "xyz")
    assembly = FiberAssembly(cell)
    random = SplitMix64(seed)
    starts, directions = [], []
    for _ in range(40):
        starts.append([side * random.unit() for _ in range(3)])
        directions.append(isotropic_direction(random))
    _straight_fibers(assembly, np.array(starts), np.array(directions), 300.0e-6, 30, 0.5 * d, 5.0 * d)
    return assembly


def _wavy_fibers(assembly, centers, directions, normals, phases, lengths, segments, diameter, min_bend_radius):
    """Planar sinusoidal waviness: offset 0.5 d sin(2 pi s / (20 d) + phase)
    along a normal perpendicular to the axis; rest shape = initial shape."""
    amplitude = 0.5 * diameter
    wavelength = 20.0 * diameter
    for center, direction, normal, phase, length in zip(centers, directions, normals, phases, lengths):
        s = (np.arange(segments + 1, dtype=np.float64) / segments - 0.5) * length
        wave = amplitude * np.sin(2.0 * math.pi * s / wavelength + phase)
        points = center[None, :] + s[:, None] * direction[None, :] + wave[:, None] * normal[None, :]
        assembly.add_fiber(points, points, radius=0.5 * diameter, min_bend_radius=min_bend_radius)


def mid_size_specimen(scale: float = 1.0, seed: int = 1, beta: float = 1.0 / 0.3,
                      fibers: int = 20000) -> FiberAssembly:
    """Periodic 2x2x2 mm cell, 20,000 fibers 1.5 mm long, diameters 7 and
    19 um split 50:50 by fiber volume (17,610 and 2,390 fibers), segment
    length 2 d (round(1.5 mm / 2 d) segments: 107 and 39), Schladitz
    orientation about z, sinusoidal waviness of amplitude 0.5 d, wavelength
    20 d and uniform phase, curvature limit 1/(5 d). About 2.0 M nodes.

    `beta` uses the Schladitz convention of
    crates/tangle_characterize/src/shape.rs:26-30 (beta = 1 isotropic, beta > 1
    lays fibers in the plane normal to the axis). The default 1/0.3 is the
    xy-biased reading of "beta = 0.3 (xy-biased)". `scale` < 1 shrinks the
    cell side by scale and the fiber count by scale**3, keeping the volume
    fraction (used for the learned-warm-start training specimens and for small
    parity cases).
    """
    side = 2.0e-3 * scale
    count = max(int(round(fibers * scale ** 3)), 2)
    ratio = (19.0 / 7.0) ** 2
    n19 = int(round(count / (1.0 + ratio)))
    n7 = count - n19
    cell = Cell([side] * 3, "xyz")
    assembly = FiberAssembly(cell)
    random = SplitMix64(seed)
    for diameter, n in ((19.0e-6, n19), (7.0e-6, n7)):
        segments = int(round(1.5e-3 / (2.0 * diameter)))
        centers, directions, normals, phases = [], [], [], []
        for _ in range(n):
            center = [side * random.unit() for _ in range(3)]
            cz = schladitz_axis_cosine_quantile(beta, random.unit())
            if random.unit() < 0.5:
                cz = -cz
            azimuth = 2.0 * math.pi * random.unit()
            sz = math.sqrt(max(1.0 - cz * cz, 0.0))
            direction = [sz * math.cos(azimuth), sz * math.sin(azimuth), cz]
            ta = perpendicular(direction)
            tb = _normalize(_cross(direction, ta))
            turn = 2.0 * math.pi * random.unit()
            normal = [math.cos(turn) * ta[i] + math.sin(turn) * tb[i] for i in range(3)]
            phase = 2.0 * math.pi * random.unit()
            centers.append(center)
            directions.append(direction)
            normals.append(normal)
            phases.append(phase)
        _wavy_fibers(assembly, np.array(centers), np.array(directions), np.array(normals), phases,
                     [1.5e-3] * n, segments, diameter, 5.0 * diameter)
    return assembly


def batched_specimens(count: int = 512, seed: int = 1, max_fibers: int = 5000) -> List[FiberAssembly]:
    """Independent specimens: fiber count log-uniform in [40, max_fibers],
    10 um fibers, length uniform in [0.3, 1] mm with segment length 2 d,
    isotropic straight fibers, periodic cube whose side gives a fiber volume
    fraction uniform in [5 %, 25 %], curvature limit 1/(5 d)."""
    d = 10.0e-6
    out = []
    for index in range(count):
        random = SplitMix64(seed * 1_000_003 + index)
        fibers = int(round(math.exp(math.log(40.0) + (math.log(max_fibers) - math.log(40.0)) * random.unit())))
        fraction = 0.05 + 0.20 * random.unit()
        lengths = [0.3e-3 + 0.7e-3 * random.unit() for _ in range(fibers)]
        volume = sum(math.pi * (0.5 * d) ** 2 * length for length in lengths)
        side = (volume / fraction) ** (1.0 / 3.0)
        side = max(side, 1.05 * max(lengths) / 2.0)
        cell = Cell([side] * 3, "xyz")
        assembly = FiberAssembly(cell)
        for length in lengths:
            segments = max(int(round(length / (2.0 * d))), 2)
            start = np.array([side * random.unit() for _ in range(3)])
            direction = np.array(isotropic_direction(random))
            steps = np.arange(segments + 1) * (length / segments)
            points = start[None, :] + steps[:, None] * direction[None, :]
            assembly.add_fiber(points, points, radius=0.5 * d, min_bend_radius=5.0 * d)
        out.append(assembly)
    return out


def _normal_deviate(random: SplitMix64) -> float:
    """Box-Muller from two unit draws (the first moved off zero)."""
    u1 = max(random.unit(), 1.0e-300)
    u2 = random.unit()
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def ply_stack_specimen(plies: int = 20, side: float = 2.0e-3, thickness: float = 0.1e-3, seed: int = 1,
                       volume_fraction: float = 0.15, fiber_length: float = 1.0e-3, segment_over_d: float = 0.8,
                       tilt_degrees: float = 3.0, rest_curvature_fraction: float = 0.5) -> FiberAssembly:
    """A stack of planar plies, each side x side x thickness, periodic in x
    and y with walls in z (the cell is plies x thickness high). Ply k holds 7
    and 19 um fibers split 50:50 by fiber volume at `volume_fraction` of the
    ply, directions uniform in the xy plane with a tilt out of it drawn from
    N(0, tilt_degrees), centres uniform in the ply; each fiber's rest (and
    initial) shape is a waviness of wavelength 20 d in a random plane through
    its axis whose peak curvature is uniform in [0, rest_curvature_fraction] x
    its limit 1/(5 d); a fiber whose tilt reaches past a wall moves along z
    until it lies inside. Segments are `segment_over_d` diameters long. Fiber f of
    ply k carries formation step k and formation layer k, so a recipe
    deposits the plies in sequence. The defaults give 20 plies of about
    146,000 segments (2.9 M segments in all)."""
    cell = Cell([side, side, plies * thickness], "xy")
    assembly = FiberAssembly(cell)
    random = SplitMix64(seed)
    ply_volume = side * side * thickness
    for k in range(plies):
        for diameter in (19.0e-6, 7.0e-6):
            radius = 0.5 * diameter
            count = max(int(round(0.5 * volume_fraction * ply_volume / (math.pi * radius * radius * fiber_length))), 1)
            segments = max(int(round(fiber_length / (segment_over_d * diameter))), 2)
            limit = 1.0 / (5.0 * diameter)
            s = (np.arange(segments + 1, dtype=np.float64) / segments - 0.5) * fiber_length
            for _ in range(count):
                azimuth = 2.0 * math.pi * random.unit()
                turn = 2.0 * math.pi * random.unit()
                peak = rest_curvature_fraction * limit * random.unit()
                phase = 2.0 * math.pi * random.unit()
                center = np.array([side * random.unit(), side * random.unit(),
                                   (k + 0.5 + 0.8 * (random.unit() - 0.5)) * thickness])
                # Waviness of wavelength 20 d whose peak curvature
                # amplitude * (2 pi / wavelength)^2 is `peak`.
                wavelength = 20.0 * diameter
                amplitude = peak * (wavelength / (2.0 * math.pi)) ** 2
                along = s
                offset = amplitude * np.sin(2.0 * math.pi * s / wavelength + phase)
                # The tilt is redrawn until the fiber fits between the walls
                # (flat after 64 draws), and the centre moves along z until
                # the whole fiber lies inside, as population.rs:657-693
                # contains a centre.
                for attempt in range(65):
                    tilt = math.radians(tilt_degrees) * _normal_deviate(random) if attempt < 64 else 0.0
                    direction = np.array([math.cos(tilt) * math.cos(azimuth), math.cos(tilt) * math.sin(azimuth),
                                          math.sin(tilt)])
                    ta = np.array(perpendicular(direction.tolist()))
                    tb = np.cross(direction, ta)
                    normal = math.cos(turn) * ta + math.sin(turn) * tb
                    shape = along[:, None] * direction[None, :] + offset[:, None] * normal[None, :]
                    low = radius - shape[:, 2].min()
                    high = plies * thickness - radius - shape[:, 2].max()
                    if low <= high:
                        break
                center[2] = min(max(center[2], low), high)
                points = center[None, :] + shape
                index = assembly.add_fiber(points, points, radius=radius, min_bend_radius=5.0 * diameter,
                                           material=f"fiber_{round(diameter * 1e6)}um")
                assembly.set_fiber_formation_step(index, k)
                assembly.set_fiber_formation_layer(index, k)
    return assembly


def layer_centers(assembly: FiberAssembly, axis: int) -> List[float]:
    """The layer targets of a layered assembly along `axis`
    (crates/tangle_generate/src/layered.rs:178-213): per formation layer
    0..max, the f64 mean of its fibers' mean vertex coordinates (serial sums),
    cast to f32. Every layer up to the largest must hold a fiber."""
    layers = [f.formation_layer for f in assembly.fibers if f.formation_layer is not None]
    if not layers:
        raise ValueError("layered formation requires formation-layer labels")
    sums = [0.0] * (max(layers) + 1)
    counts = [0] * len(sums)
    for fiber in assembly.fibers:
        if fiber.formation_layer is None:
            continue
        values = fiber.placed[:, axis].tolist()
        total = 0.0
        for value in values:
            total += value
        sums[fiber.formation_layer] += total / len(values)
        counts[fiber.formation_layer] += 1
    if min(counts) == 0:
        raise ValueError("formation layers must be contiguous and populated")
    return [float(np.float32(total / count)) for total, count in zip(sums, counts)]


def ply_collections(stack: FiberAssembly) -> List[FiberAssembly]:
    """The plies of a layered assembly as separate collections, in the
    stack's cell: collection k holds layer k's fibers in order (with their
    shapes, materials and layer labels), as a recipe inserts them one ply at
    a time."""
    layers = [f.formation_layer for f in stack.fibers if f.formation_layer is not None]
    out = [FiberAssembly(stack.cell) for _ in range(max(layers) + 1 if layers else 0)]
    for fiber in stack.fibers:
        if fiber.formation_layer is None:
            continue
        out[fiber.formation_layer].add_fiber(fiber.placed, fiber.intrinsic, radius=fiber.radius,
                                             min_bend_radius=fiber.min_bend_radius, material=fiber.material,
                                             formation_layer=fiber.formation_layer)
    return out
