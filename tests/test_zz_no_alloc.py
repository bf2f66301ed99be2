"""tgl_contact_pass_noalloc: the contact pass for callers that cannot allocate.

Some hosts hand this library only device buffers they already own -- a
solver drawing from its own fixed memory pool, or a loop that must never
wait on the allocator -- so the library may not call cudaMalloc for them.
This test gives the no-allocation entry point device arrays (allocated here
by the test, as such a caller would own them) and checks its corrections
and penetrations against the world's contact pass with neighbor capacity 1,
which takes the same exact cell scan: bit for bit, on two calls in a row
(the second call reuses the fixed scratch array the first one left behind).
"""

import ctypes

import numpy as np
import pytest

from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import cpu_runnable_specimen, mid_size_specimen
from tangle_b200.settings import CellListConfig, RelaxationSettings

pytestmark = pytest.mark.gpu


class NoallocInputs(ctypes.Structure):
    _fields_ = [
        ("positions", ctypes.c_void_p),
        ("segment_vertices", ctypes.c_void_p),
        ("segment_fibers", ctypes.c_void_p),
        ("segment_radii", ctypes.c_void_p),
        ("vertex_arc_lengths", ctypes.c_void_p),
        ("segment_count", ctypes.c_uint32),
        ("cells", ctypes.c_uint32 * 3),
        ("cell_lower", ctypes.c_float * 3),
        ("cell_upper", ctypes.c_float * 3),
        ("cell_periodic", ctypes.c_uint32 * 3),
        ("correction_fraction", ctypes.c_float),
        ("contact_aggregation", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


def arc_lengths(packed):
    """Rest arc length of every vertex (f64 accumulate, packed.rs:561-580)."""
    x = packed.intrinsic_positions.reshape(-1, 3).astype(np.float64)
    arc = np.zeros(packed.vertex_count, dtype=np.float32)
    for start, count in packed.fiber_vertex_spans.reshape(-1, 2):
        total = 0.0
        for v in range(start + 1, start + count):
            d = x[v] - x[v - 1]
            total += float(np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]))
            arc[v] = np.float32(total)
    return arc


@pytest.mark.parametrize("make", [cpu_runnable_specimen, lambda: mid_size_specimen(scale=0.25, seed=5)],
                         ids=["cpu_runnable", "mid_size_scaled"])
def test_noalloc_contact_pass_matches_the_world(make, cuda_lib):
    import torch

    from tangle_b200.device import DeviceWorld

    assembly = make()
    packed = PackedAssembly.from_assembly(assembly)
    cfg = RelaxationSettings(neighbor_capacity=1).to_config(assembly.smallest_diameter())
    world = DeviceWorld(packed, CellListConfig(neighbor_capacity=1), cfg.max_step)
    expected_corr, expected_pen = world.debug_corrections(cfg)
    dims = world.cell_dims
    world.close()

    dev = torch.device("cuda", 0)
    positions = torch.from_numpy(packed.positions.copy()).to(dev)
    seg_vertices = torch.from_numpy(packed.segment_vertices.view(np.int32).copy()).to(dev)
    seg_fibers = torch.from_numpy(packed.segment_fibers.view(np.int32).copy()).to(dev)
    radii = torch.from_numpy(packed.segment_radii.copy()).to(dev)
    arcs = torch.from_numpy(arc_lengths(packed)).to(dev)
    S = packed.segment_count
    inputs = NoallocInputs()
    inputs.positions = positions.data_ptr()
    inputs.segment_vertices = seg_vertices.data_ptr()
    inputs.segment_fibers = seg_fibers.data_ptr()
    inputs.segment_radii = radii.data_ptr()
    inputs.vertex_arc_lengths = arcs.data_ptr()
    inputs.segment_count = S
    for a in range(3):
        inputs.cells[a] = dims[a]
        inputs.cell_lower[a] = float(packed.cell_lower[a])
        inputs.cell_upper[a] = float(packed.cell_upper[a])
        inputs.cell_periodic[a] = int(packed.cell_periodic[a])
    inputs.correction_fraction = cfg.correction_fraction
    inputs.contact_aggregation = cfg.contact_aggregation

    fn = cuda_lib.tgl_contact_pass_noalloc
    fn.argtypes = [ctypes.POINTER(NoallocInputs), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        corrections = torch.full((6 * S,), float("nan"), dtype=torch.float32, device=dev)
        penetrations = torch.full((S,), float("nan"), dtype=torch.float32, device=dev)
        rc = fn(ctypes.byref(inputs), corrections.data_ptr(), penetrations.data_ptr(), stream)
        assert rc == 0, cuda_lib.tgl_last_error()
        torch.cuda.synchronize(dev)
        got_corr = corrections.cpu().numpy()
        got_pen = penetrations.cpu().numpy()
        np.testing.assert_array_equal(got_pen.view(np.uint32), expected_pen.view(np.uint32),
                                      err_msg=f"penetrations differ on call {call + 1}")
        np.testing.assert_array_equal(got_corr.view(np.uint32), expected_corr.view(np.uint32),
                                      err_msg=f"corrections differ on call {call + 1}")
    assert float(expected_pen.max()) > 0.0  # the inputs do overlap


def rejection_inputs(segments, cells):
    """Inputs whose pointers are never touched: the size checks come first."""
    inputs = NoallocInputs()
    inputs.positions = inputs.segment_vertices = inputs.segment_fibers = 1
    inputs.segment_radii = inputs.vertex_arc_lengths = 1
    inputs.segment_count = segments
    inputs.cells[:] = cells
    inputs.cell_upper[:] = [1.0, 1.0, 1.0]
    inputs.correction_fraction = 0.8
    return inputs


@pytest.mark.parametrize("segments, cells, message", [
    ((1 << 18) + 1, [1, 1, 1], b"262144 segments"),
    # 2^21 * 2^21 * 2^22 = 2^64 wraps to 0 in a 64-bit product.
    (8, [1 << 21, 1 << 21, 1 << 22], b"262144 cells"),
    (8, [1 << 22, 1 << 22, 1 << 20], b"262144 cells"),
    (8, [512, 512, 2], b"262144 cells"),
    (8, [(1 << 18) + 1, 1, 1], b"262144 cells"),
], ids=["segments", "wrapping_product", "wrapping_product_2", "product", "axis"])
def test_noalloc_rejects_inputs_beyond_its_fixed_scratch(segments, cells, message, cuda_lib):
    inputs = rejection_inputs(segments, cells)
    fn = cuda_lib.tgl_contact_pass_noalloc
    fn.argtypes = [ctypes.POINTER(NoallocInputs), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    rc = fn(ctypes.byref(inputs), 1, 1, None)
    assert rc == 5  # TGL_ERR_UNSUPPORTED, before touching any pointer or queueing anything
    cuda_lib.tgl_last_error.restype = ctypes.c_char_p
    assert message in cuda_lib.tgl_last_error()
