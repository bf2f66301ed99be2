"""ctypes binding of libtangle_cuda.so: the resident relaxation world.

`DeviceWorld` is the Python face of the reference's `DeviceWorld` seam
(crates/tangle_relax/src/device/plugin.rs:309-893) for the "cuda" backend:
`upload` (world.rs:308-690), `run_batch` (world.rs:1020-1505, returning
`BatchStatus`), `download_positions` (world.rs:2384-2390), `cell_size` /
`cell_count` (plugin.rs:597-636) and `neighbor_list_rebuilds`
(world/neighbor_list.rs:167-176). Errors from the C ABI raise
`ValueError` (invalid input) or `RuntimeError` (CUDA failure); there is no
CPU fallback: a missing library or device raises.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
import os
from typing import List, Optional

import numpy as np

from .formation import FormationHooks
from .settings import BatchStatus, CellListConfig, RelaxationConfig

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtangle_cuda.so")
_lib = None

TGL_ERR_INVALID = 1
TGL_ERR_UNSUPPORTED = 5
#: Contact-list state of a slot whose list ran past its batch's chunk.
CONTACT_USE_VERLET = 0xFFFFFFFE

#: Every symbol include/tangle_cuda.h declares.
EXPORTS = (
    "tgl_world_create", "tgl_world_destroy", "tgl_world_checkpoint", "tgl_world_restore", "tgl_run_batch",
    "tgl_arena_create", "tgl_arena_status", "tgl_capture_contacts", "tgl_download_positions", "tgl_upload_positions",
    "tgl_cell_size", "tgl_cell_count", "tgl_cell_dims", "tgl_neighbor_skin", "tgl_neighbor_block",
    "tgl_neighbor_list_rebuilds", "tgl_debug_rebuild", "tgl_debug_cell_list", "tgl_debug_neighbor_lists",
    "tgl_debug_corrections", "tgl_kernel_launches", "tgl_set_kernel_timing", "tgl_last_kernel_times",
    "tgl_world_stream", "tgl_contact_pass_noalloc", "tgl_contact_list_info", "tgl_debug_contact_lists",
    "tgl_gemm_bf16", "tgl_warmstart_graph_count", "tgl_warmstart_graph_fill", "tgl_world_displace",
    "tgl_world_residual", "tgl_mp_edge_inputs", "tgl_mp_node_inputs", "tgl_mp_node_inputs_backward",
    "tgl_mp_edge_inputs_backward", "tgl_column_sums_scratch", "tgl_column_sums", "tgl_adam_step", "tgl_mse",
    "tgl_convert_bf16", "tgl_world_set_active_fibers", "tgl_world_set_layer_targets", "tgl_world_set_vertex_targets",
    "tgl_world_vertex_target_state", "tgl_world_target_errors", "tgl_world_compact_cell", "tgl_world_cell_bounds",
    "tgl_world_compaction_metrics", "tgl_world_wall_reactions", "tgl_world_set_wall_reactions",
    "tgl_world_set_fiber_max_curvatures", "tgl_world_get_launch_params", "tgl_world_set_launch_params",
    "tgl_autotune", "tgl_warmstart_set_focus",
    "tgl_last_error",
)


class LayerTargets(ctypes.Structure):
    """tgl_layer_targets."""

    _fields_ = [
        ("axis", ctypes.c_uint32),
        ("count", ctypes.c_uint32),
        ("targets", ctypes.c_void_p),
        ("fiber_layers", ctypes.c_void_p),
        ("first_layer", ctypes.c_uint32),
        ("last_layer", ctypes.c_uint32),
        ("stiffness", ctypes.c_float),
        ("max_translation", ctypes.c_float),
        ("apply_now", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class VertexTargets(ctypes.Structure):
    """tgl_vertex_targets."""

    _fields_ = [
        ("axis", ctypes.c_uint32),
        ("count", ctypes.c_uint32),
        ("vertices", ctypes.c_void_p),
        ("displacement", ctypes.c_float),
        ("stiffness", ctypes.c_float),
        ("max_translation", ctypes.c_float),
        ("reserved", ctypes.c_uint32),
        ("coordinates", ctypes.c_void_p),
        ("command_coordinates", ctypes.c_void_p),
    ]


class Packed(ctypes.Structure):
    """tgl_packed."""

    _fields_ = [
        ("vertex_count", ctypes.c_uint32),
        ("segment_count", ctypes.c_uint32),
        ("fiber_count", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("positions", ctypes.c_void_p),
        ("intrinsic_positions", ctypes.c_void_p),
        ("segment_vertices", ctypes.c_void_p),
        ("segment_fibers", ctypes.c_void_p),
        ("segment_radii", ctypes.c_void_p),
        ("segment_rest_lengths", ctypes.c_void_p),
        ("fiber_vertex_spans", ctypes.c_void_p),
        ("fiber_segment_spans", ctypes.c_void_p),
        ("vertex_segments", ctypes.c_void_p),
        ("vertex_max_curvature", ctypes.c_void_p),
        ("vertex_pinned", ctypes.c_void_p),
        ("cell_lower", ctypes.c_float * 3),
        ("cell_upper", ctypes.c_float * 3),
        ("cell_periodic", ctypes.c_uint32 * 3),
        ("reserved2", ctypes.c_uint32),
    ]


class CellList(ctypes.Structure):
    """tgl_cell_list_config."""

    _fields_ = [
        ("cell_size_scale", ctypes.c_float),
        ("neighbor_skin_scale", ctypes.c_float),
        ("neighbor_capacity", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("max_list_bytes", ctypes.c_uint64),
    ]


class Config(ctypes.Structure):
    """tgl_relax_config."""

    _fields_ = [
        ("penetration_tolerance", ctypes.c_float),
        ("correction_fraction", ctypes.c_float),
        ("stretch_stiffness", ctypes.c_float),
        ("bend_stiffness", ctypes.c_float),
        ("curvature_limit_stiffness", ctypes.c_float),
        ("curvature_limit_safety_margin", ctypes.c_float),
        ("curvature_ratio_tolerance", ctypes.c_float),
        ("max_step", ctypes.c_float),
        ("constraint_iterations", ctypes.c_uint32),
        ("curvature_cleanup_sweeps", ctypes.c_uint32),
        ("contact_aggregation", ctypes.c_uint32),
        ("force_full_iterations", ctypes.c_uint32),
        ("motion_model", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class KernelTimes(ctypes.Structure):
    """tgl_kernel_times."""

    _fields_ = [
        ("contact_ms", ctypes.c_double),
        ("update_ms", ctypes.c_double),
        ("rebuild_ms", ctypes.c_double),
        ("contact_passes", ctypes.c_uint32),
        ("updates", ctypes.c_uint32),
        ("rebuilds", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class LaunchParams(ctypes.Structure):
    """tgl_launch_params: launch shapes that never change a result."""

    _fields_ = [
        ("lanes_per_fiber", ctypes.c_uint32),
        ("contact_blocks_per_sm", ctypes.c_uint32),
        ("build_chunk", ctypes.c_uint32),
        ("contact_skin_fraction", ctypes.c_float),
        ("update_warps_per_block", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 3),
    ]

    FIELDS = ("lanes_per_fiber", "contact_blocks_per_sm", "build_chunk", "contact_skin_fraction",
              "update_warps_per_block")
    DEFAULTS = {"update_warps_per_block": 4}  # for choices saved before the field existed

    def as_dict(self) -> dict:
        return {name: (float(getattr(self, name)) if name == "contact_skin_fraction" else int(getattr(self, name)))
                for name in self.FIELDS}

    @classmethod
    def from_dict(cls, values: dict) -> "LaunchParams":
        out = cls()
        for name in cls.FIELDS:
            setattr(out, name, values[name] if name in values else cls.DEFAULTS[name])
        return out


class AutotuneReport(ctypes.Structure):
    """tgl_autotune_report."""

    _fields_ = [
        ("trials", ctypes.c_uint32),
        ("trial_iterations", ctypes.c_uint32),
        ("default_ms", ctypes.c_float),
        ("best_ms", ctypes.c_float),
    ]


class Status(ctypes.Structure):
    """tgl_batch_status."""

    _fields_ = [
        ("total_iterations", ctypes.c_uint64),
        ("batch_iterations", ctypes.c_uint64),
        ("max_penetration", ctypes.c_float),
        ("max_displacement", ctypes.c_float),
        ("max_curvature_ratio", ctypes.c_float),
        ("converged", ctypes.c_uint32),
        ("cell_list_overflow", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


def load_library():
    """Loads the in-tree library (no fallback: raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m tangle_b200.build` (the CUDA path has no fallback)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    lib.tgl_world_create.argtypes = [ctypes.POINTER(Packed), ctypes.POINTER(CellList), ctypes.c_float,
                                     ctypes.POINTER(P)]
    lib.tgl_world_create.restype = ctypes.c_int
    lib.tgl_world_destroy.argtypes = [P]
    lib.tgl_world_destroy.restype = None
    lib.tgl_capture_contacts.argtypes = [P, ctypes.c_float, ctypes.c_uint32, P, P, P, P,
                                         ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]
    lib.tgl_capture_contacts.restype = ctypes.c_int
    lib.tgl_arena_create.argtypes = [ctypes.POINTER(Packed), ctypes.c_uint32, ctypes.POINTER(CellList), ctypes.c_float,
                                     ctypes.POINTER(ctypes.c_void_p)]
    lib.tgl_arena_create.restype = ctypes.c_int
    lib.tgl_arena_status.argtypes = [P, ctypes.POINTER(Config), ctypes.POINTER(Status), ctypes.c_uint32]
    lib.tgl_arena_status.restype = ctypes.c_int
    lib.tgl_world_checkpoint.argtypes = [P, P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)]
    lib.tgl_world_checkpoint.restype = ctypes.c_int
    lib.tgl_world_restore.argtypes = [ctypes.POINTER(Packed), ctypes.POINTER(CellList), ctypes.c_float,
                                      ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]
    lib.tgl_world_restore.restype = ctypes.c_int
    lib.tgl_run_batch.argtypes = [P, ctypes.POINTER(Config), ctypes.c_uint32, ctypes.POINTER(Status)]
    lib.tgl_run_batch.restype = ctypes.c_int
    lib.tgl_download_positions.argtypes = [P, P, ctypes.c_size_t]
    lib.tgl_download_positions.restype = ctypes.c_int
    lib.tgl_upload_positions.argtypes = [P, P, ctypes.c_size_t]
    lib.tgl_upload_positions.restype = ctypes.c_int
    lib.tgl_cell_size.argtypes = [P]
    lib.tgl_cell_size.restype = ctypes.c_float
    lib.tgl_cell_count.argtypes = [P]
    lib.tgl_cell_count.restype = ctypes.c_uint64
    lib.tgl_cell_dims.argtypes = [P, P]
    lib.tgl_cell_dims.restype = None
    lib.tgl_neighbor_skin.argtypes = [P]
    lib.tgl_neighbor_skin.restype = ctypes.c_float
    lib.tgl_neighbor_block.argtypes = [P]
    lib.tgl_neighbor_block.restype = ctypes.c_uint32
    lib.tgl_neighbor_list_rebuilds.argtypes = [P, ctypes.POINTER(ctypes.c_uint32)]
    lib.tgl_neighbor_list_rebuilds.restype = ctypes.c_int
    lib.tgl_contact_list_info.argtypes = [P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32),
                                           ctypes.POINTER(ctypes.c_uint32)]
    lib.tgl_contact_list_info.restype = ctypes.c_int
    lib.tgl_debug_contact_lists.argtypes = [P, P, P]
    lib.tgl_debug_contact_lists.restype = ctypes.c_int
    lib.tgl_debug_rebuild.argtypes = [P]
    lib.tgl_debug_rebuild.restype = ctypes.c_int
    lib.tgl_debug_cell_list.argtypes = [P, P, P, P]
    lib.tgl_debug_cell_list.restype = ctypes.c_int
    lib.tgl_debug_neighbor_lists.argtypes = [P, P, P]
    lib.tgl_debug_neighbor_lists.restype = ctypes.c_int
    lib.tgl_debug_corrections.argtypes = [P, ctypes.POINTER(Config), P, P]
    lib.tgl_debug_corrections.restype = ctypes.c_int
    lib.tgl_kernel_launches.argtypes = [P]
    lib.tgl_kernel_launches.restype = ctypes.c_uint64
    lib.tgl_world_get_launch_params.argtypes = [P, ctypes.POINTER(LaunchParams)]
    lib.tgl_world_get_launch_params.restype = ctypes.c_int
    lib.tgl_world_set_launch_params.argtypes = [P, ctypes.POINTER(LaunchParams)]
    lib.tgl_world_set_launch_params.restype = ctypes.c_int
    lib.tgl_autotune.argtypes = [P, ctypes.POINTER(Config), ctypes.c_uint32, ctypes.POINTER(LaunchParams),
                                 ctypes.POINTER(AutotuneReport)]
    lib.tgl_autotune.restype = ctypes.c_int
    lib.tgl_set_kernel_timing.argtypes = [P, ctypes.c_int]
    lib.tgl_set_kernel_timing.restype = ctypes.c_int
    lib.tgl_last_kernel_times.argtypes = [P, ctypes.POINTER(KernelTimes)]
    lib.tgl_last_kernel_times.restype = ctypes.c_int
    lib.tgl_world_stream.argtypes = [P]
    lib.tgl_world_stream.restype = ctypes.c_void_p
    lib.tgl_world_set_active_fibers.argtypes = [P, P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32),
                                                ctypes.POINTER(ctypes.c_uint32)]
    lib.tgl_world_set_layer_targets.argtypes = [P, ctypes.POINTER(LayerTargets)]
    lib.tgl_world_set_vertex_targets.argtypes = [P, ctypes.POINTER(VertexTargets)]
    lib.tgl_world_vertex_target_state.argtypes = [P, P, P, ctypes.c_uint32]
    lib.tgl_world_target_errors.argtypes = [P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32),
                                            ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32)]
    lib.tgl_world_compact_cell.argtypes = [P, P, P, ctypes.c_uint32]
    lib.tgl_world_cell_bounds.argtypes = [P, P, P]
    lib.tgl_world_compaction_metrics.argtypes = [P, ctypes.c_float, P, P]
    lib.tgl_world_wall_reactions.argtypes = [P, P, ctypes.c_size_t]
    lib.tgl_world_set_wall_reactions.argtypes = [P, P, ctypes.c_size_t]
    lib.tgl_world_set_fiber_max_curvatures.argtypes = [P, P, ctypes.c_size_t]
    for name in ("tgl_world_set_active_fibers", "tgl_world_set_layer_targets", "tgl_world_set_vertex_targets",
                 "tgl_world_vertex_target_state", "tgl_world_target_errors", "tgl_world_compact_cell",
                 "tgl_world_cell_bounds", "tgl_world_compaction_metrics", "tgl_world_wall_reactions",
                 "tgl_world_set_wall_reactions", "tgl_world_set_fiber_max_curvatures"):
        getattr(lib, name).restype = ctypes.c_int
    lib.tgl_last_error.argtypes = []
    lib.tgl_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _raise(lib, rc: int):
    message = lib.tgl_last_error().decode()
    if rc in (TGL_ERR_INVALID, TGL_ERR_UNSUPPORTED):
        raise ValueError(message)
    raise RuntimeError(f"tangle CUDA error {rc}: {message}")


def _ptr(array: Optional[np.ndarray]):
    return None if array is None else array.ctypes.data_as(ctypes.c_void_p)


def packed_struct(packed, keep: list) -> Packed:
    arrays = [
        np.ascontiguousarray(packed.positions, dtype=np.float32),
        np.ascontiguousarray(packed.intrinsic_positions, dtype=np.float32),
        np.ascontiguousarray(packed.segment_vertices, dtype=np.uint32),
        np.ascontiguousarray(packed.segment_fibers, dtype=np.uint32),
        np.ascontiguousarray(packed.segment_radii, dtype=np.float32),
        np.ascontiguousarray(packed.segment_rest_lengths, dtype=np.float32),
        np.ascontiguousarray(packed.fiber_vertex_spans, dtype=np.uint32),
        np.ascontiguousarray(packed.fiber_segment_spans, dtype=np.uint32),
        np.ascontiguousarray(packed.vertex_segments, dtype=np.uint32),
        np.ascontiguousarray(packed.vertex_max_curvature, dtype=np.float32),
        np.ascontiguousarray(packed.vertex_pinned, dtype=np.uint32),
    ]
    keep.extend(arrays)
    pk = Packed()
    pk.vertex_count = packed.vertex_count
    pk.segment_count = packed.segment_count
    pk.fiber_count = packed.fiber_count
    (pk.positions, pk.intrinsic_positions, pk.segment_vertices, pk.segment_fibers, pk.segment_radii,
     pk.segment_rest_lengths, pk.fiber_vertex_spans, pk.fiber_segment_spans, pk.vertex_segments,
     pk.vertex_max_curvature, pk.vertex_pinned) = [a.ctypes.data for a in arrays]
    for a in range(3):
        pk.cell_lower[a] = float(packed.cell_lower[a])
        pk.cell_upper[a] = float(packed.cell_upper[a])
        pk.cell_periodic[a] = int(packed.cell_periodic[a])
    return pk


def config_struct(config: RelaxationConfig) -> Config:
    return Config(
        float(config.penetration_tolerance), float(config.correction_fraction), float(config.stretch_stiffness),
        float(config.bend_stiffness), float(config.curvature_limit_stiffness),
        float(config.curvature_limit_safety_margin), float(config.curvature_ratio_tolerance),
        float(config.max_step), int(config.constraint_iterations), int(config.curvature_cleanup_sweeps),
        int(config.contact_aggregation), int(bool(config.force_full_iterations)), int(config.motion_code), 0,
    )


def cell_list_struct(cell_list: CellListConfig) -> CellList:
    return CellList(float(cell_list.cell_size_scale), float(cell_list.neighbor_skin_scale),
                    int(cell_list.neighbor_capacity), 0, int(cell_list.max_list_bytes))


@dataclass
class SegmentContactCandidate:
    """One captured contact (world.rs SegmentContactCandidate)."""

    first_segment: int
    second_segment: int
    first_coordinate: float
    second_coordinate: float
    surface_gap: float
    crossing_angle: float


@dataclass
class ContactCapture:
    candidates: List[SegmentContactCandidate]
    overflow: bool


class DeviceWorld(FormationHooks):
    """Resident relaxation world on the current CUDA device."""

    def __init__(self, packed, cell_list: Optional[CellListConfig] = None, max_step: float = 0.006,
                 total_iterations: Optional[int] = None):
        lib = load_library()
        cell_list = cell_list or CellListConfig()
        keep: list = []
        pk = packed_struct(packed, keep)
        cl = cell_list_struct(cell_list)
        handle = ctypes.c_void_p()
        if total_iterations is None:
            rc = lib.tgl_world_create(ctypes.byref(pk), ctypes.byref(cl), ctypes.c_float(max_step),
                                      ctypes.byref(handle))
        else:
            rc = lib.tgl_world_restore(ctypes.byref(pk), ctypes.byref(cl), ctypes.c_float(max_step),
                                       int(total_iterations), ctypes.byref(handle))
        if rc:
            _raise(lib, rc)
        self._lib = lib
        self._handle = handle
        self._packed = packed
        self.vertex_count = packed.vertex_count
        self.segment_count = packed.segment_count
        if not np.all(np.asarray(packed.fiber_active)):
            self.set_active_fibers(np.asarray(packed.fiber_active))

    @classmethod
    def upload(cls, config: RelaxationConfig, packed) -> "DeviceWorld":
        """DeviceWorld::upload(config, packed) (plugin.rs:422-424)."""
        return cls(packed, config.cell_list, config.max_step)

    @classmethod
    def arena(cls, packeds, cell_list: Optional[CellListConfig] = None, max_step: float = 0.006) -> "DeviceWorld":
        """tgl_arena_create: several specimens relaxed together, each with its
        own grid, lists and gate; positions are concatenated in order."""
        lib = load_library()
        cell_list = cell_list or CellListConfig()
        keep: list = []
        structs = (Packed * len(packeds))(*[packed_struct(p, keep) for p in packeds])
        cl = cell_list_struct(cell_list)
        handle = ctypes.c_void_p()
        rc = lib.tgl_arena_create(structs, len(packeds), ctypes.byref(cl), ctypes.c_float(max_step),
                                  ctypes.byref(handle))
        if rc:
            _raise(lib, rc)
        world = cls.__new__(cls)
        world._lib = lib
        world._handle = handle
        world._packed = None
        world.vertex_count = sum(p.vertex_count for p in packeds)
        world.segment_count = sum(p.segment_count for p in packeds)
        world.specimen_vertices = [p.vertex_count for p in packeds]
        return world

    def capture_contacts(self, maximum_surface_gap: float, capacity: int) -> "ContactCapture":
        """DeviceWorld::capture_contacts (world.rs:2195-2335): current
        inter-fiber contacts within the gap, sorted."""
        segments = np.empty(2 * capacity, dtype=np.uint32)
        coordinates = np.empty(2 * capacity, dtype=np.float32)
        gaps = np.empty(capacity, dtype=np.float32)
        angles = np.empty(capacity, dtype=np.float32)
        count, overflow = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self._lib.tgl_capture_contacts(self._handle, ctypes.c_float(maximum_surface_gap), int(capacity),
                                                   _ptr(segments), _ptr(coordinates), _ptr(gaps), _ptr(angles),
                                                   ctypes.byref(count), ctypes.byref(overflow)))
        n = int(count.value)
        candidates = [SegmentContactCandidate(int(segments[2 * i]), int(segments[2 * i + 1]),
                                              float(coordinates[2 * i]), float(coordinates[2 * i + 1]),
                                              float(gaps[i]), float(angles[i])) for i in range(n)]
        return ContactCapture(candidates, bool(overflow.value))

    def specimen_statuses(self, config: RelaxationConfig) -> List[BatchStatus]:
        """tgl_arena_status: each specimen's status after the last batch."""
        n = len(self.specimen_vertices)
        out = (Status * n)()
        self._check(self._lib.tgl_arena_status(self._handle, ctypes.byref(config_struct(config)), out, n))
        return [BatchStatus(total_iterations=int(st.total_iterations), batch_iterations=int(st.batch_iterations),
                            max_penetration=float(st.max_penetration), max_displacement=float(st.max_displacement),
                            max_curvature_ratio=float(st.max_curvature_ratio), converged=bool(st.converged),
                            cell_list_overflow=bool(st.cell_list_overflow)) for st in out]

    def specimen_positions(self) -> List[np.ndarray]:
        """The arena's positions split per specimen (interleaved xyz each)."""
        xyz = self.download_positions()
        bounds = np.cumsum([0] + [3 * v for v in self.specimen_vertices])
        return [xyz[a:b] for a, b in zip(bounds[:-1], bounds[1:])]

    @classmethod
    def restore(cls, config: RelaxationConfig, checkpoint) -> "DeviceWorld":
        """DeviceWorld::restore(config, checkpoint) (plugin.rs:358-391;
        world.rs:693-756): a world uploaded from the checkpoint's packed
        assembly (positions, cell, active fibers, curvature limits) whose
        lifetime iteration count continues from the checkpoint's, with its
        wall reactions and formation targets re-installed."""
        world = cls(checkpoint.packed, config.cell_list, config.max_step, checkpoint.total_iterations)
        world._restore_formation(checkpoint)
        return world

    def checkpoint(self):
        """DeviceWorld::checkpoint() (plugin.rs:393-404; world.rs:758-823):
        the packed assembly with the current positions, cell, active fibers
        and curvature limits, the lifetime iteration count, the wall
        reactions and the installed formation targets."""
        import dataclasses

        from .checkpoint import DeviceWorldCheckpoint

        xyz = np.empty(3 * self.vertex_count, dtype=np.float32)
        total = ctypes.c_uint64()
        self._check(self._lib.tgl_world_checkpoint(self._handle, _ptr(xyz), xyz.size, ctypes.byref(total)))
        lower, upper = self._fh_cell_bounds()
        packed = dataclasses.replace(self._packed, positions=xyz, cell_lower=lower, cell_upper=upper,
                                     fiber_active=self.fiber_active, vertex_max_curvature=self.vertex_max_curvature)
        return DeviceWorldCheckpoint(packed, int(total.value), self.wall_reactions(), self.layer_target_checkpoint(),
                                     self.vertex_target_checkpoint())

    # ---- formation hooks (tangle_b200.formation.FormationHooks)

    def _fh_set_active(self, flags):
        segments, vertices = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self._lib.tgl_world_set_active_fibers(self._handle, _ptr(flags), flags.size,
                                                          ctypes.byref(segments), ctypes.byref(vertices)))
        return int(segments.value), int(vertices.value)

    def _fh_set_layer_targets(self, axis, targets, layers, first, last, stiffness, max_translation, apply_now):
        if targets is None:
            self._check(self._lib.tgl_world_set_layer_targets(self._handle, None))
            return
        t = LayerTargets(axis, targets.size, targets.ctypes.data, layers.ctypes.data, first, last, stiffness,
                         max_translation, 1 if apply_now else 0, 0)
        self._check(self._lib.tgl_world_set_layer_targets(self._handle, ctypes.byref(t)))

    def _fh_set_vertex_targets(self, axis, indices, displacement, stiffness, max_translation, coordinates, commands):
        if indices is None:
            self._check(self._lib.tgl_world_set_vertex_targets(self._handle, None))
            return
        t = VertexTargets(axis, indices.size, indices.ctypes.data, displacement, stiffness, max_translation, 0,
                          None if coordinates is None else coordinates.ctypes.data,
                          None if commands is None else commands.ctypes.data)
        self._check(self._lib.tgl_world_set_vertex_targets(self._handle, ctypes.byref(t)))

    def _fh_vertex_target_state(self, count):
        coordinates = np.empty(count, dtype=np.float32)
        commands = np.empty(count, dtype=np.float32)
        self._check(self._lib.tgl_world_vertex_target_state(self._handle, _ptr(coordinates), _ptr(commands), count))
        return coordinates, commands

    def _fh_target_errors(self):
        layer, vertex = ctypes.c_float(), ctypes.c_float()
        has_layer, has_vertex = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self._lib.tgl_world_target_errors(self._handle, ctypes.byref(layer), ctypes.byref(has_layer),
                                                      ctypes.byref(vertex), ctypes.byref(has_vertex)))
        return float(layer.value), bool(has_layer.value), float(vertex.value), bool(has_vertex.value)

    def _fh_compact(self, lower, upper, kinematics):
        self._check(self._lib.tgl_world_compact_cell(self._handle, _ptr(lower), _ptr(upper), kinematics))

    def _fh_cell_bounds(self):
        lower = np.empty(3, dtype=np.float32)
        upper = np.empty(3, dtype=np.float32)
        self._check(self._lib.tgl_world_cell_bounds(self._handle, _ptr(lower), _ptr(upper)))
        return lower, upper

    def _fh_metrics(self, correction_fraction, stiffness):
        out = np.empty(13, dtype=np.float32)
        self._check(self._lib.tgl_world_compaction_metrics(self._handle, ctypes.c_float(correction_fraction),
                                                           _ptr(stiffness), _ptr(out)))
        return out

    def _fh_wall_reactions(self):
        out = np.empty(3 * self.vertex_count, dtype=np.float32)
        self._check(self._lib.tgl_world_wall_reactions(self._handle, _ptr(out), out.size))
        return out

    def _fh_set_wall_reactions(self, xyz):
        self._check(self._lib.tgl_world_set_wall_reactions(self._handle, _ptr(xyz), xyz.size))

    def _fh_set_fiber_curvatures(self, values):
        self._check(self._lib.tgl_world_set_fiber_max_curvatures(self._handle, _ptr(values), values.size))

    def packed(self):
        """DeviceWorld::packed() (plugin.rs:619-636): the uploaded host assembly."""
        return self._packed

    def close(self) -> None:
        if getattr(self, "_handle", None):
            self._lib.tgl_world_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc:
            _raise(self._lib, rc)

    def run_batch(self, config: RelaxationConfig, iterations: int) -> BatchStatus:
        st = Status()
        self._check(self._lib.tgl_run_batch(self._handle, ctypes.byref(config_struct(config)), int(iterations),
                                            ctypes.byref(st)))
        return BatchStatus(
            total_iterations=int(st.total_iterations),
            batch_iterations=int(st.batch_iterations),
            max_penetration=float(st.max_penetration),
            max_displacement=float(st.max_displacement),
            max_curvature_ratio=float(st.max_curvature_ratio),
            converged=bool(st.converged),
            cell_list_overflow=bool(st.cell_list_overflow),
        )

    def download_positions(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(3 * self.vertex_count, dtype=np.float32)
        self._check(self._lib.tgl_download_positions(self._handle, _ptr(out), out.size))
        return out

    def upload_positions(self, positions) -> None:
        arr = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
        self._check(self._lib.tgl_upload_positions(self._handle, _ptr(arr), arr.size))

    @property
    def cell_size(self) -> float:
        return float(self._lib.tgl_cell_size(self._handle))

    @property
    def cell_count(self) -> int:
        return int(self._lib.tgl_cell_count(self._handle))

    @property
    def cell_dims(self):
        dims = np.zeros(3, dtype=np.uint32)
        self._lib.tgl_cell_dims(self._handle, _ptr(dims))
        return tuple(int(v) for v in dims)

    @property
    def neighbor_skin(self) -> float:
        return float(self._lib.tgl_neighbor_skin(self._handle))

    @property
    def neighbor_block(self) -> int:
        return int(self._lib.tgl_neighbor_block(self._handle))

    @property
    def kernel_launches(self) -> int:
        return int(self._lib.tgl_kernel_launches(self._handle))

    @property
    def stream_handle(self) -> int:
        """The cudaStream_t (as an int) this world's kernels run on."""
        return int(self._lib.tgl_world_stream(self._handle) or 0)

    def launch_params(self) -> dict:
        """The launch shapes in use (tgl_world_get_launch_params)."""
        out = LaunchParams()
        self._check(self._lib.tgl_world_get_launch_params(self._handle, ctypes.byref(out)))
        return out.as_dict()

    def set_launch_params(self, params: dict) -> None:
        """Applies launch shapes (tgl_world_set_launch_params); results do
        not change."""
        self._check(self._lib.tgl_world_set_launch_params(self._handle, ctypes.byref(LaunchParams.from_dict(params))))

    def autotune_trials(self, config: RelaxationConfig, trial_iterations: int = 32):
        """tgl_autotune: searches the launch shapes on this world's current
        state (which it leaves as it found it) and applies the fastest.
        Returns (params, report)."""
        best = LaunchParams()
        report = AutotuneReport()
        self._check(self._lib.tgl_autotune(self._handle, ctypes.byref(config_struct(config)), int(trial_iterations),
                                           ctypes.byref(best), ctypes.byref(report)))
        return best.as_dict(), {"trials": int(report.trials), "trial_iterations": int(report.trial_iterations),
                                "default_ms": float(report.default_ms), "best_ms": float(report.best_ms)}

    def set_kernel_timing(self, enable: bool) -> None:
        self._check(self._lib.tgl_set_kernel_timing(self._handle, 1 if enable else 0))

    def last_kernel_times(self) -> dict:
        t = KernelTimes()
        self._check(self._lib.tgl_last_kernel_times(self._handle, ctypes.byref(t)))
        return {"contact_ms": t.contact_ms, "update_ms": t.update_ms, "rebuild_ms": t.rebuild_ms,
                "contact_passes": t.contact_passes, "updates": t.updates, "steps": t.rebuilds}

    def neighbor_list_rebuilds(self) -> int:
        out = ctypes.c_uint32()
        self._check(self._lib.tgl_neighbor_list_rebuilds(self._handle, ctypes.byref(out)))
        return int(out.value)

    def contact_list_info(self) -> dict:
        """Contact-list skin (0 when off), entries per slot and refreshes so far."""
        skin = ctypes.c_float()
        block = ctypes.c_uint32()
        refreshes = ctypes.c_uint32()
        self._check(self._lib.tgl_contact_list_info(self._handle, ctypes.byref(skin), ctypes.byref(block),
                                                    ctypes.byref(refreshes)))
        return {"skin": float(skin.value), "block": int(block.value), "refreshes": int(refreshes.value)}

    def debug_contact_states(self) -> np.ndarray:
        """The contact-list state of every cell-list slot [S]: its list length,
        CONTACT_USE_VERLET or 0xFFFFFFFF (tgl_debug_contact_lists without the
        chunks)."""
        states = np.empty(self.segment_count, dtype=np.uint32)
        self._check(self._lib.tgl_debug_contact_lists(self._handle, _ptr(states), None))
        return states

    def debug_contact_lists(self):
        """Contact lists by cell-list slot: counts [S] and a list per slot.
        A list of None (count CONTACT_USE_VERLET) marks a slot whose list ran
        past its batch's chunk (its contact pass reads the Verlet list); an
        empty list with count 0 also stands for a slot whose Verlet list
        overflowed (it scans the cells). Unpacked from the per-batch chunks
        tgl_debug_contact_lists returns."""
        block = self.contact_list_info()["block"]
        S = self.segment_count
        states = np.empty(S, dtype=np.uint32)
        chunks = np.empty(max((S + 31) // 32 * 32 * block, 1), dtype=np.uint32)
        self._check(self._lib.tgl_debug_contact_lists(self._handle, _ptr(states), _ptr(chunks)))
        counts = np.zeros(S, dtype=np.uint32)
        out = []
        for base in range(0, S, 32):
            at = base * block
            for slot in range(base, min(S, base + 32)):
                state = int(states[slot])
                if state == 0xFFFFFFFF:
                    out.append(np.empty(0, dtype=np.uint32))
                elif state == CONTACT_USE_VERLET:
                    counts[slot] = CONTACT_USE_VERLET
                    out.append(None)
                else:
                    counts[slot] = state
                    out.append(chunks[at: at + state].copy())
                    at += state
        return counts, out

    def debug_rebuild(self) -> None:
        self._check(self._lib.tgl_debug_rebuild(self._handle))

    def debug_cell_list(self):
        C = self.cell_count
        counts = np.empty(C, dtype=np.uint32)
        offsets = np.empty(C, dtype=np.uint32)
        segments = np.empty(self.segment_count, dtype=np.uint32)
        self._check(self._lib.tgl_debug_cell_list(self._handle, _ptr(counts), _ptr(offsets), _ptr(segments)))
        return counts, offsets, segments

    def debug_neighbor_lists_raw(self):
        """Verlet lists as stored: true counts [S] and the block-strided list
        array [block * S] (entries past a count, or of a segment whose count
        exceeds the block, are unspecified)."""
        block = self.neighbor_block
        counts = np.empty(self.segment_count, dtype=np.uint32)
        lists = np.empty(max(block * self.segment_count, 1), dtype=np.uint32)
        self._check(self._lib.tgl_debug_neighbor_lists(self._handle, _ptr(counts), _ptr(lists)))
        return counts, lists

    def debug_neighbor_lists(self):
        block = self.neighbor_block
        counts = np.empty(self.segment_count, dtype=np.uint32)
        lists = np.empty(max(block * self.segment_count, 1), dtype=np.uint32)
        self._check(self._lib.tgl_debug_neighbor_lists(self._handle, _ptr(counts), _ptr(lists)))
        out = []
        for s in range(self.segment_count):
            n = int(counts[s])
            out.append(lists[block * s: block * s + n].copy() if n <= block else None)
        return counts, out

    def debug_corrections(self, config: RelaxationConfig):
        corr = np.empty(6 * self.segment_count, dtype=np.float32)
        pen = np.empty(self.segment_count, dtype=np.float32)
        self._check(self._lib.tgl_debug_corrections(self._handle, ctypes.byref(config_struct(config)), _ptr(corr),
                                                    _ptr(pen)))
        return corr, pen
