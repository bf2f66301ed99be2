"""Rigid-translation motion (kernels.rs:1539-1646) and the contact
aggregations 1 (penetration weighted) and 2 (deepest only,
contact.rs:844-870).

* The reference's known answer world_tests.rs:787-834: the crossed pair
  relaxed by rigid translation converges within 20 iterations and keeps
  every fiber's centerline vector to 1e-6 (oracle and CUDA).
* Parity: positions after 7 + 13 iterations bit-identical between the CUDA
  path and the oracle, and the same iteration and rebuild counts, for
  rigid motion and for each aggregation, on four specimens.
"""

import numpy as np
import pytest

import fixtures as fx
from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import cpu_runnable_specimen, mid_size_specimen
from tangle_b200.settings import CellListConfig, RelaxationConfig

from test_known_answers import BACKENDS, make_world


@pytest.mark.parametrize("kind", BACKENDS)
def test_rigid_translation_preserves_centerline_vectors(kind, request):
    if kind == "cuda":
        request.getfixturevalue("cuda_lib")
    assembly = fx.crossed_assembly()
    packed = PackedAssembly.from_assembly(assembly)
    before = packed.positions.reshape(-1, 6)
    vectors = before[:, 3:] - before[:, :3]
    w = make_world(kind, assembly, 0.2)
    config = RelaxationConfig(motion_model="rigid_translation", penetration_tolerance=1.0e-5,
                              correction_fraction=1.0, max_step=0.2, max_iterations=20, iterations_per_batch=20)
    status = w.run_batch(config, 20)
    assert status.converged
    after = w.download_positions().reshape(-1, 6)
    np.testing.assert_allclose(after[:, 3:] - after[:, :3], vectors, atol=1.0e-6)


def specimens():
    c1 = cpu_runnable_specimen(seed=4)
    small = mid_size_specimen(scale=0.15, seed=6)
    return [
        ("cpu_runnable", c1, RelaxationConfig(penetration_tolerance=1.0e-8, max_step=0.6e-6)),
        ("mid_size_scaled", small, RelaxationConfig(penetration_tolerance=7.0e-9, max_step=0.4e-6,
                                                    cell_list=CellListConfig(neighbor_capacity=256,
                                                                             max_list_bytes=1 << 30))),
        ("dense_mat", fx.dense_crossed_mat(), RelaxationConfig(penetration_tolerance=0.0, max_step=0.01)),
        ("hairpin_walls", fx.hairpin(), RelaxationConfig(penetration_tolerance=1.0e-4, max_step=0.02)),
    ]


SPECIMENS = specimens()
VARIANTS = [("rigid", {"motion_model": "rigid_translation"}), ("weighted", {"contact_aggregation": 1}),
            ("deepest", {"contact_aggregation": 2}),
            ("rigid_deepest", {"motion_model": "rigid_translation", "contact_aggregation": 2})]


@pytest.mark.gpu
@pytest.mark.parametrize("variant", VARIANTS, ids=[v[0] for v in VARIANTS])
@pytest.mark.parametrize("case", SPECIMENS, ids=[c[0] for c in SPECIMENS])
def test_cuda_matches_the_oracle_bit_for_bit(case, variant, cuda_lib):
    from oracle import OracleWorld
    from tangle_b200.device import DeviceWorld

    name, assembly, base = case
    cfg = RelaxationConfig(**{**base.__dict__, **variant[1], "force_full_iterations": True})
    packed = PackedAssembly.from_assembly(assembly)
    orc = OracleWorld(packed, cfg.cell_list, cfg.max_step)
    dev = DeviceWorld(packed, cfg.cell_list, cfg.max_step)
    for batch in (7, 13):
        so = orc.run_batch(cfg, batch)
        sd = dev.run_batch(cfg, batch)
        assert (so.total_iterations, so.batch_iterations) == (sd.total_iterations, sd.batch_iterations)
        assert np.float32(so.max_penetration) == np.float32(sd.max_penetration)
        assert np.float32(so.max_displacement) == np.float32(sd.max_displacement)
    po, pd = orc.download_positions(), dev.download_positions()
    np.testing.assert_array_equal(po.view(np.uint32), pd.view(np.uint32), err_msg=f"{name} {variant[0]}")
    assert orc.neighbor_list_rebuilds() == dev.neighbor_list_rebuilds()
