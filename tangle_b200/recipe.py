"""`Recipe` / `RunResult`: the reference's Python entry point to relaxation
and formation.

Mirrors crates/tangle_python/python/tangle/_tangle.pyi:898-1014 and
crates/tangle_python/src/recipe.rs:240-560 for the recording side, and the
run loop of crates/tangle_python/src/recipe.rs:618-723 with the batch
controller of crates/tangle_relax/src/device/plugin.rs:1041-1181 and the
formation operations of crates/tangle_generate/src/recipe.rs:859-1600:

* every `insert` is a formation step: the whole recipe's fibers are uploaded
  once and the step's fibers join the resident world when the step is
  reached (activate_formation_step, no re-upload);
* unset length settings are sized from the smallest fiber diameter;
* a recipe that only inserts fibers relaxes them until converged;
* each batch runs at most `iterations_per_batch` iterations and at most the
  run-wide `max_iterations` remaining; `relax_for` and `settle_targets`
  force full batches;
* layer operations hold layer targets on the stack axis (`scale_layer_spacing`,
  `place_layer_above`) until `release_layer_placement` or the end of the
  recipe; `needle_layer` pulls chosen fibers of a layer through the stack
  with vertex displacement targets until `release_needles`;
  `fit_cell_to_active_fibers` moves the walls onto the active fibers;
  `set_min_bend_radius` changes a material's curvature limit;
* a step that exhausts its budget raises `RecipeError`.
"""

from __future__ import annotations

import copy
from dataclasses import dataclass
from typing import List, Optional, Sequence, Union

import numpy as np

from . import checkpoint as ckpt
from .assembly import Cell, FiberAssembly, Material, PackedAssembly
from .checkpoint import CheckpointReport, CheckpointSettings
from .device import DeviceWorld
from .formation import CompactionKinematics
from .generate import FiberPopulation, generate_fiber_population, layer_centers
from .needling import (CircularFootprint, NeedlingConfig, RandomFiberFraction, random_footprint_center,
                       selected_needling_vertices)
from .settings import BatchStatus, RelaxationSettings

DEFAULT_STACK_AXIS = 2


class RecipeError(RuntimeError):
    """A recorded step could not be completed (_tangle.pyi:38)."""

    def __init__(self, operation: int, description: str, iteration: int, reason: str):
        super().__init__(f"operation {operation} ({description}) failed at iteration {iteration}: {reason}")
        self.operation = operation
        self.description = description
        self.iteration = iteration
        self.reason = reason


@dataclass
class FiberSelection:
    """The fibers one `insert` added (recipe.rs PyFiberSelection): their
    indices in the recipe's assembly and their formation step."""

    name: str
    fibers: List[int]
    formation_step: int


class HeldTargets:
    """Returned by operations that hold fibers on targets (_tangle.pyi:898-913):
    as a context manager it records the matching release when the block ends."""

    def __init__(self, recipe: "Recipe", release):
        self._recipe = recipe
        self._release = release

    def __enter__(self) -> "Recipe":
        return self._recipe

    def __exit__(self, exc_type=None, exc=None, traceback=None) -> bool:
        self._release()
        return False


@dataclass
class _Insert:
    step: int
    count: int


@dataclass
class _RelaxUntilConverged:
    maximum_iterations: int


@dataclass
class _RelaxFor:
    iterations: int


@dataclass
class _SettleTargets:
    tolerance: float
    maximum_iterations: int


@dataclass
class _SetMinBendRadius:
    material: str
    minimum_bend_radius: float


@dataclass
class _ScaleLayerSpacing:
    factor: float
    stiffness: float
    max_translation: float


@dataclass
class _PlaceLayerAbove:
    layer: int
    gap: float
    stiffness: float
    max_translation: float


@dataclass
class _ReleaseLayerPlacement:
    pass


@dataclass
class _FitCell:
    axes: List[bool]
    padding: float


@dataclass
class _NeedleLayer:
    config: NeedlingConfig


@dataclass
class _ReleaseNeedles:
    pass


class RunResult:
    """The relaxed fibers and run statistics (_tangle.pyi:1003-1014)."""

    def __init__(self, assembly: FiberAssembly, status: BatchStatus, uploaded_bytes: int, downloaded_bytes: int,
                 cell_size: float, cell_count: int, rebuilds: int, report: Optional[CheckpointReport] = None,
                 events: Optional[List[str]] = None):
        self.assembly = assembly
        self._status = status
        self.uploaded_bytes = uploaded_bytes
        self.downloaded_bytes = downloaded_bytes
        self.cell_size = cell_size
        self.cell_count = cell_count
        self.neighbor_list_rebuilds = rebuilds
        self.events = list(events or [])
        report = report or CheckpointReport()
        self.resumed = report.resumed
        self.resumed_iteration = report.resumed_iteration
        self.checkpoint_saves = report.saves
        self.last_checkpoint_iteration = report.last_saved_iteration
        self.last_checkpoint_bytes = report.last_saved_bytes

    fiber_count = property(lambda self: self.assembly.fiber_count)
    iterations = property(lambda self: self._status.total_iterations)
    converged = property(lambda self: self._status.converged)
    max_penetration = property(lambda self: self._status.max_penetration)
    max_curvature_ratio = property(lambda self: self._status.max_curvature_ratio)
    max_displacement = property(lambda self: self._status.max_displacement)

    def centerlines(self) -> List[List[List[float]]]:
        return self.assembly.centerlines()

    def __repr__(self) -> str:
        return (f"RunResult(fibers={self.fiber_count}, iterations={self.iterations}, converged={self.converged}, "
                f"max_penetration={self.max_penetration:.3e}, max_curvature_ratio={self.max_curvature_ratio:.6f})")


def _upload_bytes(packed: PackedAssembly) -> int:
    arrays = [packed.positions, packed.intrinsic_positions, packed.segment_vertices, packed.segment_fibers,
              packed.segment_radii, packed.segment_rest_lengths, packed.fiber_vertex_spans,
              packed.fiber_segment_spans, packed.vertex_segments, packed.vertex_max_curvature, packed.vertex_pinned]
    return int(sum(a.nbytes for a in arrays)) + 6 * 4 + 3 * 4


def infer_stack_axis(periodic: Sequence[bool]) -> int:
    """collection.rs:104-112: z unless it is periodic, else the last walled axis."""
    if not periodic[DEFAULT_STACK_AXIS]:
        return DEFAULT_STACK_AXIS
    for axis in (2, 1, 0):
        if not periodic[axis]:
            return axis
    return DEFAULT_STACK_AXIS


def _positive(value: float, name: str) -> float:
    value = float(value)
    if not (np.isfinite(value) and value > 0.0):
        raise ValueError(f"{name} must be positive and finite")
    return value


def _unit_fraction(value: float, name: str) -> float:
    value = float(value)
    if not (0.0 < value <= 1.0):
        raise ValueError(f"{name} must be in (0, 1]")
    return value


def active_capsule_bounds(packed: PackedAssembly, positions: np.ndarray, fiber_active: np.ndarray,
                          padding: float):
    """compaction_control.rs:446-474: the box around every active segment's
    capsule (its endpoints grown by its radius plus `padding`), in f32."""
    active = np.asarray(fiber_active, dtype=bool)[np.asarray(packed.segment_fibers)]
    if not np.any(active):
        raise ValueError("cannot fit a cell without active fiber segments")
    xyz = np.asarray(positions, dtype=np.float32).reshape(-1, 3)
    ends = np.asarray(packed.segment_vertices).reshape(-1, 2)[active]
    grow = (np.asarray(packed.segment_radii, dtype=np.float32)[active] + np.float32(padding))[:, None]
    lower = np.minimum((xyz[ends[:, 0]] - grow).min(axis=0), (xyz[ends[:, 1]] - grow).min(axis=0))
    upper = np.maximum((xyz[ends[:, 0]] + grow).max(axis=0), (xyz[ends[:, 1]] + grow).max(axis=0))
    return lower.astype(np.float32), upper.astype(np.float32)


class Recipe:
    """An ordered list of steps on one cell; nothing runs until `run`."""

    def __init__(self, cell: Union[Cell, FiberAssembly], *, stack_axis: Optional[int] = None):
        if isinstance(cell, FiberAssembly):
            self._assembly = copy.deepcopy(cell)
        elif isinstance(cell, Cell):
            self._assembly = FiberAssembly(cell)
        else:
            raise TypeError("Recipe needs a Cell or a FiberAssembly")
        if stack_axis is None:
            stack_axis = infer_stack_axis(self._assembly.cell.periodic)
        if stack_axis not in (0, 1, 2):
            raise ValueError("stack_axis must be 0, 1 or 2")
        self._stack_axis = int(stack_axis)
        self._operations: list = []
        self._descriptions: List[str] = []
        self._next_step = 0

    @property
    def cell(self) -> Cell:
        return self._assembly.cell

    @property
    def stack_axis(self) -> int:
        return self._stack_axis

    def _push(self, operation, description: str) -> None:
        self._operations.append(operation)
        self._descriptions.append(description)

    def insert(self, collection, *, name: Optional[str] = None, translation: Sequence[float] = (0.0, 0.0, 0.0),
               rotation: Optional[Sequence[Sequence[float]]] = None) -> FiberSelection:
        """recipe.rs:249-296: the collection's fibers, rotated then
        translated, become the next formation step."""
        if isinstance(collection, FiberPopulation):
            collection = generate_fiber_population(self._assembly.cell, collection)
        if not isinstance(collection, FiberAssembly):
            raise TypeError("insert takes a FiberAssembly (a generated collection) or a FiberPopulation")
        if not collection.fibers:
            raise ValueError("cannot insert an empty fiber collection")
        rotation = np.eye(3) if rotation is None else np.asarray(rotation, dtype=np.float64)
        translation = np.asarray(translation, dtype=np.float64)
        if rotation.shape != (3, 3) or translation.shape != (3,):
            raise ValueError("rotation must be 3x3 and translation three values")
        step = self._next_step
        self._next_step += 1
        indices = []
        for fiber in collection.fibers:
            index = self._assembly.add_fiber(fiber.placed @ rotation.T + translation,
                                             fiber.intrinsic @ rotation.T + translation, radius=fiber.radius,
                                             min_bend_radius=fiber.min_bend_radius, material=fiber.material,
                                             formation_layer=fiber.formation_layer)
            self._assembly.set_fiber_formation_step(index, step)
            indices.append(index)
        name = name or "collection"
        self._push(_Insert(step, len(indices)),
                   f"insert {name!r} ({len(indices)} fibers) as formation step {step}")
        return FiberSelection(name, indices, step)

    def relax_until_converged(self, *, max_iterations: int = 2000) -> None:
        if max_iterations <= 0:
            raise ValueError("max_iterations must be positive")
        self._push(_RelaxUntilConverged(int(max_iterations)), "relax until converged")

    def relax_for(self, iterations: int) -> None:
        if iterations <= 0:
            raise ValueError("iterations must be positive")
        self._push(_RelaxFor(int(iterations)), f"relax for {iterations} iterations")

    def settle_targets(self, *, tolerance: float, max_iterations: int) -> None:
        """recipe.rs:328-342: relax in full batches until every held target
        is within `tolerance`."""
        tolerance = float(tolerance)
        if not (np.isfinite(tolerance) and tolerance >= 0.0):
            raise ValueError("tolerance must be non-negative and finite")
        if max_iterations <= 0:
            raise ValueError("max_iterations must be positive")
        self._push(_SettleTargets(tolerance, int(max_iterations)), f"settle held targets to tolerance {tolerance}")

    def set_min_bend_radius(self, material: Union[Material, str], min_bend_radius: float) -> None:
        """recipe.rs:366-394: every fiber of `material` takes this bend limit."""
        name = material.name if isinstance(material, Material) else material
        if not isinstance(name, str):
            raise TypeError("material must be a Material or a material name")
        if not name.strip():
            raise ValueError("material name must not be empty")
        radius = _positive(min_bend_radius, "min_bend_radius")
        self._push(_SetMinBendRadius(name, radius), f"set {name!r} minimum bend radius to {radius:.3e}")

    def scale_layer_spacing(self, factor: float, *, stiffness: float = 0.25,
                            max_translation: float = 1.0e-5) -> HeldTargets:
        """recipe.rs:396-415 (MoveLayers): every layer's target moves to the
        cell centre plus `factor` times its initial offset."""
        self._push(_ScaleLayerSpacing(_positive(factor, "factor"), _unit_fraction(stiffness, "stiffness"),
                                      _positive(max_translation, "max_translation")),
                   f"scale layer spacing by {factor}")
        return HeldTargets(self, self.release_layer_placement)

    def place_layer_above(self, layer: int, *, gap: float, stiffness: float = 0.25,
                          max_translation: float = 1.0e-5) -> HeldTargets:
        """recipe.rs:419-443 (PlaceLayerAbove): layer `layer` is held `gap`
        above layer `layer - 1`'s target."""
        if int(layer) <= 0:
            raise ValueError("layer must be greater than zero")
        self._push(_PlaceLayerAbove(int(layer), _positive(gap, "gap"), _unit_fraction(stiffness, "stiffness"),
                                    _positive(max_translation, "max_translation")),
                   f"place layer {layer} above layer {int(layer) - 1}")
        return HeldTargets(self, self.release_layer_placement)

    def release_layer_placement(self) -> None:
        self._push(_ReleaseLayerPlacement(), "release layer placement")

    def needle_layer(self, layer: int, *, footprint, depth: float, min_fiber_diameter: Optional[float] = None,
                     stiffness: float = 0.25, max_translation: float = 1.0e-5,
                     max_translation_over_diameter: float = 0.25) -> HeldTargets:
        """recipe.rs:455-503 (NeedleLayer): fibers of `layer` chosen by the
        footprint are each pulled at one internal vertex `depth` toward the
        negative stack axis, held until `release_needles`."""
        depth = _positive(depth, "depth")
        if min_fiber_diameter is not None:
            min_fiber_diameter = _positive(min_fiber_diameter, "min_fiber_diameter")
        stiffness = _unit_fraction(stiffness, "stiffness")
        max_translation = _positive(max_translation, "max_translation")
        ratio = _positive(max_translation_over_diameter, "max_translation_over_diameter")
        layer = int(layer)
        if isinstance(footprint, RandomFiberFraction):
            how = f"a random {footprint.fraction} of its fibers"
        elif isinstance(footprint, CircularFootprint):
            if footprint.center is None:  # recipe.rs:761-776: a reproducible centre per layer
                plane = [a for a in range(3) if a != self._stack_axis]
                cell = self._assembly.cell
                center = random_footprint_center(footprint.seed, layer, [cell.origin[a] for a in plane],
                                                 [cell.lengths[a] for a in plane])
                footprint = CircularFootprint(center, diameter=footprint.diameter)
            how = f"a {footprint.diameter:.3e} circle at [{footprint.center[0]:.3e}, {footprint.center[1]:.3e}]"
        else:
            raise TypeError("footprint must be a CircularFootprint or RandomFiberFraction")
        config = NeedlingConfig(layer, footprint, depth, stiffness, max_translation, ratio, min_fiber_diameter)
        self._push(_NeedleLayer(config), f"needle layer {layer} through {how}")
        return HeldTargets(self, self.release_needles)

    def release_needles(self) -> None:
        self._push(_ReleaseNeedles(), "release needles")

    def fit_cell_to_active_fibers(self, *, axes: Optional[Sequence[bool]] = None, padding: float = 0.0) -> None:
        """recipe.rs:515-545 (FitCellToActiveFibers): the walls of the chosen
        axes (the stack axis by default) move onto the active fibers."""
        if axes is None:
            axes = [axis == self._stack_axis for axis in range(3)]
        axes = [bool(a) for a in axes]
        if len(axes) != 3 or not any(axes):
            raise ValueError("at least one cell-fit axis must be selected")
        padding = float(padding)
        if not (np.isfinite(padding) and padding >= 0.0):
            raise ValueError("padding must be non-negative and finite")
        for axis in range(3):
            if axes[axis] and self._assembly.cell.periodic[axis]:
                raise ValueError(f"cannot fit periodic cell axis {axis} to active fibers")
        self._push(_FitCell(axes, padding), f"fit cell to active fibers with {padding:.3e} padding")

    def operations(self) -> List[str]:
        return list(self._descriptions)

    def centerlines(self) -> List[List[List[float]]]:
        return self._assembly.centerlines()

    def run(self, settings: Optional[RelaxationSettings] = None, *,
            checkpoint: Optional[CheckpointSettings] = None, world_factory=None) -> RunResult:
        """Simulates every recorded step and returns the relaxed fibers.

        With `checkpoint`, the run saves a restart file whenever the lifetime
        iteration count crosses a multiple of `interval_iterations` and when
        it ends; with `checkpoint.resume` it first restores the world and the
        recipe's progress from `resume_path` (or `path`), or only the world
        when `fresh_formation_on_resume` (tangle_checkpoint lib.rs:214-345).
        `world_factory(packed, cell_list, max_step)` replaces the CUDA world
        (tests drive the oracle through it).
        """
        if not self._assembly.fibers:
            raise ValueError("recipe contains no fibers")
        if not self._operations:
            raise ValueError("recipe contains no operations")
        settings = settings or RelaxationSettings()
        if settings.backend != "cuda":
            raise ValueError(f"backend={settings.backend!r} belongs to the reference implementation; "
                             "this library provides backend='cuda'")
        config = settings.to_config(self._assembly.smallest_diameter())
        operations = list(self._operations)
        descriptions = list(self._descriptions)
        if all(isinstance(op, _Insert) for op in operations):
            operations.append(_RelaxUntilConverged(config.max_iterations))
            descriptions.append("relax until converged")
        assembly = copy.deepcopy(self._assembly)
        axis = self._stack_axis
        status = BatchStatus(max_penetration=float("inf"), max_curvature_ratio=float("inf"))
        report = CheckpointReport()
        events: List[str] = []
        first_operation, first_completed = 0, 0
        packed = PackedAssembly.from_assembly(assembly, config.pin_fiber_ends)
        uploaded = _upload_bytes(packed)
        factory = world_factory or (lambda p, cl, step: DeviceWorld(p, cl, step))
        world = None
        if checkpoint is not None and checkpoint.resume:
            source = checkpoint.resume_path or checkpoint.path
            saved = ckpt.load(source, checkpoint.resume_case_id or checkpoint.case_id)
            sp = saved.device.packed
            if (sp.fiber_count, sp.vertex_count, sp.segment_count) != (packed.fiber_count, packed.vertex_count,
                                                                       packed.segment_count):
                raise ckpt.CheckpointError("checkpoint assembly does not match the recipe's fibers")
            if world_factory is not None:
                raise ValueError("a resumed run restores the CUDA world")
            world = DeviceWorld.restore(config, saved.device)
            packed = sp
            status = BatchStatus(total_iterations=saved.device.total_iterations, max_penetration=float("inf"),
                                 max_curvature_ratio=float("inf"))
            if not checkpoint.fresh_formation_on_resume:
                first_operation, first_completed = saved.operation, saved.operation_iterations
                status.converged = saved.converged
            report.resumed = True
            report.resumed_iteration = saved.device.total_iterations
            report.last_saved_iteration = saved.device.total_iterations
        else:
            world = factory(packed, config.cell_list, config.max_step)
        downloaded = 0
        initial_targets: List[float] = []
        current_targets: List[float] = []

        def save(index: int, completed: int, terminal: bool) -> None:
            nonlocal downloaded
            if checkpoint is None:
                return
            iteration = status.total_iterations
            if iteration == 0 or report.last_saved_iteration == iteration:
                return
            if not terminal and not ckpt.crossed_interval(iteration, report.last_saved_iteration,
                                                          checkpoint.interval_iterations):
                return
            state = world.checkpoint()
            downloaded += state.packed.positions.nbytes + 8
            size = ckpt.save(checkpoint.path, ckpt.RunCheckpoint(checkpoint.case_id, state, index, completed,
                                                                   status.converged))
            report.saves += 1
            report.last_saved_iteration = iteration
            report.last_saved_bytes = size

        def relax(index: int, budget: int, force: bool, done) -> None:
            """Batches until done() or the budget is spent (then RecipeError
            unless the step is a fixed interval)."""
            nonlocal status, downloaded
            started = status.total_iterations - (first_completed if index == first_operation else 0)
            while True:
                completed = status.total_iterations - started
                if done():
                    return
                if completed >= budget:
                    if force and not isinstance(operations[index], _SettleTargets):
                        return
                    raise RecipeError(index, descriptions[index], status.total_iterations, failure(budget))
                remaining = config.max_iterations - status.total_iterations
                if remaining <= 0:
                    raise RecipeError(index, descriptions[index], status.total_iterations,
                                      "run-wide max_iterations exhausted")
                batch = min(remaining, config.iterations_per_batch, budget - completed)
                batch_config = copy.copy(config)
                batch_config.force_full_iterations = config.force_full_iterations or force
                status = world.run_batch(batch_config, batch)
                downloaded += 11 * 4 + 3 * 4
                if status.cell_list_overflow:
                    save(index, status.total_iterations - started, True)
                    raise RecipeError(index, descriptions[index], status.total_iterations, "cell list overflow")
                save(index, status.total_iterations - started, False)

        def failure(budget: int) -> str:
            op = operations[current]
            if isinstance(op, _SettleTargets):
                error = world.formation_target_error()
                worst = max(v for v in (error.layer, error.vertex) if v is not None)
                return (f"formation targets remained at residual {worst:.3e} after {budget} iterations "
                        f"(tolerance {op.tolerance:.3e})")
            return (f"failed to converge in {budget} iterations: penetration {status.max_penetration:.3e}, "
                    f"curvature ratio {status.max_curvature_ratio:.6f}")

        def ensure_layer_targets() -> None:
            if not initial_targets:
                initial_targets.extend(layer_centers(assembly, axis))
                current_targets.extend(initial_targets)

        current = 0
        try:
            for index, op in enumerate(operations):
                current = index
                if index < first_operation:
                    continue
                if isinstance(op, _Insert):
                    # recipe.rs:925-946: the step's fibers join the resident world.
                    world.activate_formation_step(op.step)
                    status.converged = False
                elif isinstance(op, (_RelaxUntilConverged, _RelaxFor)):
                    force = isinstance(op, _RelaxFor)
                    budget = op.iterations if force else op.maximum_iterations
                    relax(index, budget, force, lambda: not force and status.converged)
                    if force:
                        status.converged = False
                elif isinstance(op, _SettleTargets):
                    def settled(op=op):
                        error = world.formation_target_error()
                        values = [v for v in (error.layer, error.vertex) if v is not None]
                        return not values or max(values) <= op.tolerance
                    relax(index, op.maximum_iterations, True, settled)
                    status.converged = False
                elif isinstance(op, _SetMinBendRadius):
                    # recipe.rs:947-1007.
                    matching = [i for i, f in enumerate(assembly.fibers) if f.material == op.material]
                    if not matching:
                        known = sorted({f.material for f in assembly.fibers if f.material is not None})
                        raise RecipeError(index, descriptions[index], status.total_iterations,
                                          f"unknown material {op.material!r}; known materials: {known}")
                    for i in matching:
                        assembly.fibers[i].min_bend_radius = op.minimum_bend_radius
                    limits = np.array([0.0 if f.min_bend_radius is None else np.float32(1.0 / f.min_bend_radius)
                                       for f in assembly.fibers], dtype=np.float32)
                    world.set_fiber_maximum_curvatures(limits)
                    status.converged = False
                elif isinstance(op, _ScaleLayerSpacing):
                    # recipe.rs:1008-1046 (MoveLayers).
                    ensure_layer_targets()
                    lower = np.float64(assembly.cell.origin[axis])
                    center = np.float32(lower + 0.5 * assembly.cell.lengths[axis])
                    current_targets[:] = [float(center + (np.float32(t) - center) * np.float32(op.factor))
                                          for t in initial_targets]
                    world.apply_layer_targets(axis, current_targets, op.stiffness, op.max_translation)
                    status.converged = False
                elif isinstance(op, _PlaceLayerAbove):
                    # recipe.rs:1047-1085.
                    ensure_layer_targets()
                    if op.layer >= len(current_targets):
                        raise RecipeError(index, descriptions[index], status.total_iterations,
                                          f"cannot place layer {op.layer}: only {len(current_targets)} layers exist")
                    current_targets[op.layer] = float(np.float32(current_targets[op.layer - 1]) + np.float32(op.gap))
                    world.apply_single_layer_target(axis, current_targets, op.layer, op.stiffness,
                                                    op.max_translation)
                    status.converged = False
                elif isinstance(op, _ReleaseLayerPlacement):
                    world.clear_layer_targets()
                    status.converged = False
                elif isinstance(op, _NeedleLayer):
                    # recipe.rs:1086-1180.
                    cfg = op.config
                    active = np.asarray(world.fiber_active, dtype=bool)
                    steps = np.asarray(packed.fiber_formation_steps)
                    active_step = int(steps[active].max()) if np.any(active) else None
                    if active_step is None or active_step < cfg.layer:
                        raise RecipeError(index, descriptions[index], status.total_iterations,
                                          f"cannot needle layer {cfg.layer}: it has not been inserted yet")
                    positions = world.download_positions()
                    downloaded += positions.nbytes
                    vertices = selected_needling_vertices(assembly, packed, positions, active, active_step, axis, cfg)
                    world.clear_vertex_targets()
                    if vertices:
                        spans = np.asarray(packed.fiber_vertex_spans).reshape(-1, 2)
                        fibers = np.searchsorted(spans[:, 0], np.asarray(vertices), side="right") - 1
                        smallest = min(2.0 * assembly.fibers[int(f)].radius for f in fibers)
                        limit = np.float32(smallest) * np.float32(cfg.max_translation_over_diameter)
                        world.apply_vertex_displacement_targets(axis, vertices, -cfg.depth, cfg.stiffness,
                                                                float(min(np.float32(cfg.max_translation), limit)))
                    events_detail = f" ({len(vertices)} vertices)"
                    descriptions[index] = descriptions[index] + events_detail
                    status.converged = False
                elif isinstance(op, _ReleaseNeedles):
                    world.clear_vertex_targets()
                    status.converged = False
                elif isinstance(op, _FitCell):
                    # recipe.rs:1205-1255: walls onto the active capsules.
                    positions = world.download_positions()
                    downloaded += positions.nbytes
                    old_lower, old_upper = world.cell_bounds()
                    fiber_lower, fiber_upper = active_capsule_bounds(packed, positions, world.fiber_active,
                                                                     op.padding)
                    new_lower = [max(float(fiber_lower[a]), old_lower[a]) if op.axes[a] else old_lower[a]
                                 for a in range(3)]
                    new_upper = [min(float(fiber_upper[a]), old_upper[a]) if op.axes[a] else old_upper[a]
                                 for a in range(3)]
                    world.compact_cell(new_lower, new_upper, CompactionKinematics.MOVING_WALLS)
                    lower, upper = world.cell_bounds()
                    assembly.cell = Cell([u - l for l, u in zip(lower, upper)], assembly.cell.periodic, lower)
                    status.converged = False
                events.append(descriptions[index])
            # recipe.rs:905-921: the recipe ends with its targets released.
            world.clear_layer_targets()
            world.clear_vertex_targets()
            save(len(operations), 0, True)
            positions = world.download_positions()
            downloaded += positions.nbytes
            world.unpack_positions(positions, assembly)
            return RunResult(assembly, status, uploaded, downloaded, world.cell_size, world.cell_count,
                             world.neighbor_list_rebuilds(), report, events)
        finally:
            close = getattr(world, "close", None)
            if close is not None:
                close()
