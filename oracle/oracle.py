"""ctypes front end of the CPU oracle (relax_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by `__graft_entry__.smoke()`
and by bench.py's CPU-baseline and reference legs, never by the product
package. `OracleWorld` exposes the same calls as the product's
`tangle_b200.DeviceWorld` so parity tests drive both the same way.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

from tangle_b200.formation import FormationHooks

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compiles liboracle.so with the committed Makefile (when missing or
    older than its sources)."""
    sources = [os.path.join(_HERE, name) for name in ("relax_oracle.cpp", "relax_oracle.h", "Makefile")]
    stale = not os.path.exists(_LIB_PATH) or any(
        os.path.exists(p) and os.path.getmtime(p) > os.path.getmtime(_LIB_PATH) for p in sources)
    if force or stale:
        subprocess.run(["make", "-C", _HERE, "CXX=g++"], check=True, capture_output=True)
    return _LIB_PATH


class _Packed(ctypes.Structure):
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


class _CellList(ctypes.Structure):
    _fields_ = [
        ("cell_size_scale", ctypes.c_float),
        ("neighbor_skin_scale", ctypes.c_float),
        ("neighbor_capacity", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("max_list_bytes", ctypes.c_uint64),
    ]


class _Config(ctypes.Structure):
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


class _Status(ctypes.Structure):
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


def _load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    lib.orc_world_create.argtypes = [ctypes.POINTER(_Packed), ctypes.POINTER(_CellList), ctypes.c_float, ctypes.POINTER(P)]
    lib.orc_world_create.restype = ctypes.c_int
    lib.orc_world_destroy.argtypes = [P]
    lib.orc_run_batch.argtypes = [P, ctypes.POINTER(_Config), ctypes.c_uint32, ctypes.POINTER(_Status)]
    lib.orc_run_batch.restype = ctypes.c_int
    lib.orc_download_positions.argtypes = [P, P, ctypes.c_size_t]
    lib.orc_upload_positions.argtypes = [P, P, ctypes.c_size_t]
    lib.orc_cell_size.argtypes = [P]
    lib.orc_cell_size.restype = ctypes.c_float
    lib.orc_cell_count.argtypes = [P]
    lib.orc_cell_count.restype = ctypes.c_uint64
    lib.orc_cell_dims.argtypes = [P, P]
    lib.orc_neighbor_skin.argtypes = [P]
    lib.orc_neighbor_skin.restype = ctypes.c_float
    lib.orc_neighbor_block.argtypes = [P]
    lib.orc_neighbor_block.restype = ctypes.c_uint32
    lib.orc_neighbor_list_rebuilds.argtypes = [P]
    lib.orc_neighbor_list_rebuilds.restype = ctypes.c_uint32
    lib.orc_set_threads.argtypes = [ctypes.c_int]
    lib.orc_debug_cell_list.argtypes = [P, P, P, P]
    lib.orc_debug_neighbor_lists.argtypes = [P, P, P]
    lib.orc_debug_corrections.argtypes = [P, ctypes.POINTER(_Config), P, P]
    lib.orc_debug_rebuild.argtypes = [P]
    lib.orc_set_active_fibers.argtypes = [P, P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32),
                                          ctypes.POINTER(ctypes.c_uint32)]
    lib.orc_set_layer_targets.argtypes = [P, ctypes.c_uint32, P, ctypes.c_uint32, P, ctypes.c_uint32,
                                          ctypes.c_uint32, ctypes.c_float, ctypes.c_float, ctypes.c_int]
    lib.orc_set_vertex_targets.argtypes = [P, ctypes.c_uint32, P, ctypes.c_uint32, ctypes.c_float, ctypes.c_float,
                                           ctypes.c_float]
    lib.orc_vertex_target_state.argtypes = [P, P, P, ctypes.c_uint32]
    lib.orc_target_errors.argtypes = [P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32)]
    lib.orc_compact_cell.argtypes = [P, P, P, ctypes.c_uint32]
    lib.orc_cell_bounds.argtypes = [P, P, P]
    lib.orc_compaction_metrics.argtypes = [P, ctypes.c_float, P, P]
    lib.orc_wall_reactions.argtypes = [P, P, ctypes.c_size_t]
    lib.orc_set_fiber_max_curvatures.argtypes = [P, P, ctypes.c_size_t]
    lib.orc_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def set_threads(threads: int) -> None:
    _load().orc_set_threads(int(threads))


def _ptr(array: Optional[np.ndarray]):
    return None if array is None else array.ctypes.data_as(ctypes.c_void_p)


class OracleWorld(FormationHooks):
    """The oracle's resident world: upload, run_batch, download, and the
    formation hooks of tangle_b200.formation."""

    def __init__(self, packed, cell_list=None, max_step: float = 0.006):
        from tangle_b200.settings import CellListConfig

        lib = _load()
        cell_list = cell_list or CellListConfig()
        self._keep = [
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
        k = self._keep
        pk = _Packed()
        pk.vertex_count = packed.vertex_count
        pk.segment_count = packed.segment_count
        pk.fiber_count = packed.fiber_count
        (pk.positions, pk.intrinsic_positions, pk.segment_vertices, pk.segment_fibers, pk.segment_radii,
         pk.segment_rest_lengths, pk.fiber_vertex_spans, pk.fiber_segment_spans, pk.vertex_segments,
         pk.vertex_max_curvature, pk.vertex_pinned) = [a.ctypes.data for a in k]
        for a in range(3):
            pk.cell_lower[a] = float(packed.cell_lower[a])
            pk.cell_upper[a] = float(packed.cell_upper[a])
            pk.cell_periodic[a] = int(packed.cell_periodic[a])
        cl = _CellList(
            float(cell_list.cell_size_scale), float(cell_list.neighbor_skin_scale),
            int(cell_list.neighbor_capacity), 0, int(cell_list.max_list_bytes),
        )
        handle = ctypes.c_void_p()
        if lib.orc_world_create(ctypes.byref(pk), ctypes.byref(cl), ctypes.c_float(max_step), ctypes.byref(handle)):
            raise ValueError(lib.orc_last_error().decode())
        self._handle = handle
        self._lib = lib
        self._packed = packed
        self.vertex_count = packed.vertex_count
        self.segment_count = packed.segment_count
        self._keep = None
        if not np.all(np.asarray(packed.fiber_active)):
            self.set_active_fibers(np.asarray(packed.fiber_active))

    def _call(self, rc: int) -> None:
        if rc:
            raise ValueError(self._lib.orc_last_error().decode())

    # ---- formation hooks (tangle_b200.formation.FormationHooks)

    def _fh_set_active(self, flags):
        segments, vertices = ctypes.c_uint32(), ctypes.c_uint32()
        self._call(self._lib.orc_set_active_fibers(self._handle, _ptr(flags), flags.size, ctypes.byref(segments),
                                                   ctypes.byref(vertices)))
        return int(segments.value), int(vertices.value)

    def _fh_set_layer_targets(self, axis, targets, layers, first, last, stiffness, max_translation, apply_now):
        count = 0 if targets is None else targets.size
        self._call(self._lib.orc_set_layer_targets(self._handle, axis, _ptr(targets), count, _ptr(layers), first, last,
                                                   stiffness, max_translation, 1 if apply_now else 0))

    def _fh_set_vertex_targets(self, axis, indices, displacement, stiffness, max_translation, coordinates, commands):
        if coordinates is not None:
            raise ValueError("the oracle installs vertex targets from the positions only")
        count = 0 if indices is None else indices.size
        self._call(self._lib.orc_set_vertex_targets(self._handle, axis, _ptr(indices), count, displacement, stiffness,
                                                    max_translation))

    def _fh_vertex_target_state(self, count):
        coordinates = np.empty(count, dtype=np.float32)
        commands = np.empty(count, dtype=np.float32)
        self._call(self._lib.orc_vertex_target_state(self._handle, _ptr(coordinates), _ptr(commands), count))
        return coordinates, commands

    def _fh_target_errors(self):
        layer, vertex = ctypes.c_float(), ctypes.c_float()
        has_layer, has_vertex = ctypes.c_uint32(), ctypes.c_uint32()
        self._call(self._lib.orc_target_errors(self._handle, ctypes.byref(layer), ctypes.byref(has_layer),
                                               ctypes.byref(vertex), ctypes.byref(has_vertex)))
        return float(layer.value), bool(has_layer.value), float(vertex.value), bool(has_vertex.value)

    def _fh_compact(self, lower, upper, kinematics):
        self._call(self._lib.orc_compact_cell(self._handle, _ptr(lower), _ptr(upper), kinematics))

    def _fh_cell_bounds(self):
        lower = np.empty(3, dtype=np.float32)
        upper = np.empty(3, dtype=np.float32)
        self._call(self._lib.orc_cell_bounds(self._handle, _ptr(lower), _ptr(upper)))
        return lower, upper

    def _fh_metrics(self, correction_fraction, stiffness):
        out = np.empty(13, dtype=np.float32)
        self._call(self._lib.orc_compaction_metrics(self._handle, ctypes.c_float(correction_fraction), _ptr(stiffness),
                                                    _ptr(out)))
        return out

    def _fh_wall_reactions(self):
        out = np.empty(3 * self.vertex_count, dtype=np.float32)
        self._call(self._lib.orc_wall_reactions(self._handle, _ptr(out), out.size))
        return out

    def _fh_set_wall_reactions(self, xyz):
        raise ValueError("the oracle does not restore wall reactions")

    def _fh_set_fiber_curvatures(self, values):
        self._call(self._lib.orc_set_fiber_max_curvatures(self._handle, _ptr(values), values.size))

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.orc_world_destroy(self._handle)
            self._handle = None

    def __del__(self):
        self.close()

    def run_batch(self, config, iterations: int):
        from tangle_b200.settings import BatchStatus

        c = _config(config)
        st = _Status()
        if self._lib.orc_run_batch(self._handle, ctypes.byref(c), int(iterations), ctypes.byref(st)):
            raise ValueError(self._lib.orc_last_error().decode())
        return BatchStatus(
            total_iterations=int(st.total_iterations),
            batch_iterations=int(st.batch_iterations),
            max_penetration=float(st.max_penetration),
            max_displacement=float(st.max_displacement),
            max_curvature_ratio=float(st.max_curvature_ratio),
            converged=bool(st.converged),
            cell_list_overflow=bool(st.cell_list_overflow),
        )

    def download_positions(self) -> np.ndarray:
        out = np.empty(3 * self.vertex_count, dtype=np.float32)
        self._lib.orc_download_positions(self._handle, _ptr(out), out.size)
        return out

    def upload_positions(self, positions) -> None:
        arr = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
        if arr.size != 3 * self.vertex_count:
            raise ValueError("position buffer has the wrong length")
        self._lib.orc_upload_positions(self._handle, _ptr(arr), arr.size)

    @property
    def cell_size(self) -> float:
        return float(self._lib.orc_cell_size(self._handle))

    @property
    def cell_count(self) -> int:
        return int(self._lib.orc_cell_count(self._handle))

    @property
    def cell_dims(self):
        dims = np.zeros(3, dtype=np.uint32)
        self._lib.orc_cell_dims(self._handle, _ptr(dims))
        return tuple(int(v) for v in dims)

    @property
    def neighbor_skin(self) -> float:
        return float(self._lib.orc_neighbor_skin(self._handle))

    @property
    def neighbor_block(self) -> int:
        return int(self._lib.orc_neighbor_block(self._handle))

    def neighbor_list_rebuilds(self) -> int:
        return int(self._lib.orc_neighbor_list_rebuilds(self._handle))

    def debug_rebuild(self) -> None:
        self._lib.orc_debug_rebuild(self._handle)

    def debug_cell_list(self):
        C = self.cell_count
        counts = np.empty(C, dtype=np.uint32)
        offsets = np.empty(C, dtype=np.uint32)
        segments = np.empty(self.segment_count, dtype=np.uint32)
        self._lib.orc_debug_cell_list(self._handle, _ptr(counts), _ptr(offsets), _ptr(segments))
        return counts, offsets, segments

    def debug_neighbor_lists_raw(self):
        """Verlet lists as stored: true counts [S] and the block-strided list
        array [block * S] (entries past a count, or of a segment whose count
        exceeds the block, are unspecified)."""
        block = self.neighbor_block
        counts = np.empty(self.segment_count, dtype=np.uint32)
        lists = np.empty(max(block * self.segment_count, 1), dtype=np.uint32)
        self._lib.orc_debug_neighbor_lists(self._handle, _ptr(counts), _ptr(lists))
        return counts, lists

    def debug_neighbor_lists(self):
        block = self.neighbor_block
        counts = np.empty(self.segment_count, dtype=np.uint32)
        lists = np.empty(max(block * self.segment_count, 1), dtype=np.uint32)
        self._lib.orc_debug_neighbor_lists(self._handle, _ptr(counts), _ptr(lists))
        out = []
        for s in range(self.segment_count):
            n = int(counts[s])
            out.append(lists[block * s : block * s + n].copy() if n <= block else None)
        return counts, out

    def debug_corrections(self, config):
        c = _config(config)
        corr = np.empty(6 * self.segment_count, dtype=np.float32)
        pen = np.empty(self.segment_count, dtype=np.float32)
        self._lib.orc_debug_corrections(self._handle, ctypes.byref(c), _ptr(corr), _ptr(pen))
        return corr, pen


def _config(config) -> _Config:
    return _Config(
        float(config.penetration_tolerance), float(config.correction_fraction), float(config.stretch_stiffness),
        float(config.bend_stiffness), float(config.curvature_limit_stiffness),
        float(config.curvature_limit_safety_margin), float(config.curvature_ratio_tolerance),
        float(config.max_step), int(config.constraint_iterations), int(config.curvature_cleanup_sweeps),
        int(config.contact_aggregation), int(bool(config.force_full_iterations)), int(config.motion_code), 0,
    )
