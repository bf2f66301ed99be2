"""`Recipe` / `RunResult`: the reference's Python entry point to relaxation.

Mirrors crates/tangle_python/python/tangle/_tangle.pyi:915-1014 for the
relaxation operations, and the run loop of
crates/tangle_python/src/recipe.rs:618-723 with the batch controller of
crates/tangle_relax/src/device/plugin.rs:1041-1181 and the operation
controllers of crates/tangle_generate/src/recipe.rs:1311-1380:

* unset length settings are sized from the smallest fiber diameter;
* a recipe that only inserts fibers relaxes them until converged;
* each batch runs at most `iterations_per_batch` iterations and at most the
  run-wide `max_iterations` remaining; `relax_for` forces full batches;
* a `relax_until_converged` step that exhausts its budget raises
  `RecipeError`.
"""

from __future__ import annotations

import copy
from dataclasses import dataclass
from typing import List, Optional, Union

import numpy as np

from . import checkpoint as ckpt
from .assembly import Cell, FiberAssembly, PackedAssembly
from .checkpoint import CheckpointReport, CheckpointSettings
from .device import DeviceWorld
from .generate import FiberPopulation, generate_fiber_population
from .settings import BatchStatus, RelaxationSettings


class RecipeError(RuntimeError):
    """A recorded step could not be completed (_tangle.pyi:38)."""

    def __init__(self, operation: int, description: str, iteration: int, reason: str):
        super().__init__(f"operation {operation} ({description}) failed at iteration {iteration}: {reason}")
        self.operation = operation
        self.description = description
        self.iteration = iteration
        self.reason = reason


@dataclass
class _Insert:
    assembly: FiberAssembly
    count: int = 0  # fibers this step adds


@dataclass
class _RelaxUntilConverged:
    maximum_iterations: int


@dataclass
class _RelaxFor:
    iterations: int


class RunResult:
    """The relaxed fibers and run statistics (_tangle.pyi:1003-1014)."""

    def __init__(self, assembly: FiberAssembly, status: BatchStatus, uploaded_bytes: int, downloaded_bytes: int,
                 cell_size: float, cell_count: int, rebuilds: int, report: Optional[CheckpointReport] = None):
        self.assembly = assembly
        self._status = status
        self.uploaded_bytes = uploaded_bytes
        self.downloaded_bytes = downloaded_bytes
        self.cell_size = cell_size
        self.cell_count = cell_count
        self.neighbor_list_rebuilds = rebuilds
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


class Recipe:
    """An ordered list of steps on one cell; nothing runs until `run`."""

    def __init__(self, cell: Union[Cell, FiberAssembly]):
        if isinstance(cell, FiberAssembly):
            self._assembly = copy.deepcopy(cell)
        elif isinstance(cell, Cell):
            self._assembly = FiberAssembly(cell)
        else:
            raise TypeError("Recipe needs a Cell or a FiberAssembly")
        self._operations: list = []
        self._descriptions: List[str] = []

    @property
    def cell(self) -> Cell:
        return self._assembly.cell

    def insert(self, collection) -> None:
        if isinstance(collection, FiberPopulation):
            collection = generate_fiber_population(self._assembly.cell, collection)
        if not isinstance(collection, FiberAssembly):
            raise TypeError("insert takes a FiberAssembly (a generated collection) or a FiberPopulation")
        for fiber in collection.fibers:
            self._assembly.add_fiber(fiber.placed, fiber.intrinsic, radius=fiber.radius,
                                     min_bend_radius=fiber.min_bend_radius)
        self._operations.append(_Insert(collection, collection.fiber_count))
        self._descriptions.append(f"insert {collection.fiber_count} fibers")

    def relax_until_converged(self, *, max_iterations: int = 2000) -> None:
        if max_iterations <= 0:
            raise ValueError("max_iterations must be positive")
        self._operations.append(_RelaxUntilConverged(int(max_iterations)))
        self._descriptions.append("relax until converged")

    def relax_for(self, iterations: int) -> None:
        if iterations <= 0:
            raise ValueError("iterations must be positive")
        self._operations.append(_RelaxFor(int(iterations)))
        self._descriptions.append(f"relax for {iterations} iterations")

    def operations(self) -> List[str]:
        return list(self._descriptions)

    def centerlines(self) -> List[List[List[float]]]:
        return self._assembly.centerlines()

    def run(self, settings: Optional[RelaxationSettings] = None, *,
            checkpoint: Optional[CheckpointSettings] = None) -> RunResult:
        """Simulates every recorded step and returns the relaxed fibers.

        With `checkpoint`, the run saves a restart file whenever the lifetime
        iteration count crosses a multiple of `interval_iterations` and when
        it ends; with `checkpoint.resume` it first restores the world and the
        recipe's progress from `resume_path` (or `path`), or only the world
        when `fresh_formation_on_resume` (tangle_checkpoint lib.rs:214-345).
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
        # Staged activation (kernels.rs:164-221): the fibers of an insert step
        # take part from that step on. The world holds the fibers active so
        # far; when a relaxation step follows new inserts, it is re-created
        # from the relaxed positions plus the new fibers (the lifetime
        # iteration count carries over). Lists only need to be supersets of
        # the contacts, so this moves nothing differently from masking.
        active_after, active = [], 0
        for op in operations:
            if isinstance(op, _Insert):
                active += op.count
            active_after.append(active)
        status = BatchStatus(max_penetration=float("inf"), max_curvature_ratio=float("inf"))
        report = CheckpointReport()
        first_operation, first_completed = 0, 0
        world, world_fibers, packed, uploaded = None, 0, None, 0

        def first_fibers(k: int) -> FiberAssembly:
            sub = FiberAssembly(assembly.cell)
            for fiber in assembly.fibers[:k]:
                sub.add_fiber(fiber.placed, fiber.intrinsic, radius=fiber.radius,
                              min_bend_radius=fiber.min_bend_radius)
            return sub

        def activate(k: int) -> None:
            nonlocal world, world_fibers, packed, uploaded
            if world is not None:
                if k == world_fibers:
                    return
                packed.unpack_positions(world.download_positions(), assembly)
                world.close()
            packed = PackedAssembly.from_assembly(first_fibers(k), config.pin_fiber_ends)
            world = DeviceWorld(packed, config.cell_list, config.max_step,
                                status.total_iterations if status.total_iterations else None)
            uploaded += _upload_bytes(packed)
            world_fibers = k

        if checkpoint is not None and checkpoint.resume:
            source = checkpoint.resume_path or checkpoint.path
            saved = ckpt.load(source, checkpoint.resume_case_id or checkpoint.case_id)
            k = saved.device.packed.fiber_count
            expected = PackedAssembly.from_assembly(first_fibers(k), config.pin_fiber_ends) if k <= len(
                assembly.fibers) else None
            if expected is None or saved.device.packed.vertex_count != expected.vertex_count or \
                    saved.device.packed.segment_count != expected.segment_count:
                raise ckpt.CheckpointError("checkpoint assembly does not match the recipe's fibers")
            world = DeviceWorld.restore(config, saved.device)
            packed = saved.device.packed
            world_fibers = k
            uploaded += _upload_bytes(packed)
            status = BatchStatus(total_iterations=saved.device.total_iterations, max_penetration=float("inf"),
                                 max_curvature_ratio=float("inf"))
            if not checkpoint.fresh_formation_on_resume:
                first_operation, first_completed = saved.operation, saved.operation_iterations
                status.converged = saved.converged
            report.resumed = True
            report.resumed_iteration = saved.device.total_iterations
            report.last_saved_iteration = saved.device.total_iterations
        downloaded = 0

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

        try:
            for index, op in enumerate(operations):
                if isinstance(op, _Insert) or index < first_operation:
                    continue
                activate(active_after[index])
                started = status.total_iterations - (first_completed if index == first_operation else 0)
                force = isinstance(op, _RelaxFor)
                budget = op.iterations if force else op.maximum_iterations
                while True:
                    completed = status.total_iterations - started
                    if not force and status.converged:
                        break
                    if completed >= budget:
                        if force:
                            break
                        raise RecipeError(index, descriptions[index], status.total_iterations,
                                          f"failed to converge in {budget} iterations: penetration "
                                          f"{status.max_penetration:.3e}, curvature ratio "
                                          f"{status.max_curvature_ratio:.6f}")
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
                if force:
                    status.converged = False
            if world is None:  # nothing to relax: the fibers stay where they were placed
                activate(active_after[-1])
            save(len(operations), 0, True)
            positions = world.download_positions()
            downloaded += positions.nbytes
            packed.unpack_positions(positions, assembly)
            return RunResult(assembly, status, uploaded, downloaded, world.cell_size, world.cell_count,
                             world.neighbor_list_rebuilds(), report)
        finally:
            if world is not None:
                world.close()
