"""bench.py prints one workload description in both arms (the GPU batch and
the CPU reference arm). It is computed from the seeded system sizes and the
mesh rule, so it must agree with the systems the GPU step builds and with
the meshes the oracle's planner gives them (the same rule as the library's
planner)."""
import numpy as np
import pytest

import bench
from esp_hoomd_b200 import systems
from oracle import esp_port as EP


def test_workload_description_matches_the_batch():
    for count in (32, 256):
        cfg = bench.workload_config(count, 1)
        sl = bench._systems(0, count)
        assert cfg["systems_per_gpu"] == count == len(sl)
        assert cfg["particles_per_gpu"] == sum(s.N for s in sl)
        prm = EP.plan(sl, bench.RCUT)
        assert cfg["mesh_points_per_gpu"] == sum(int(np.prod(p.mesh)) for p in prm)
    # the batch is the published mixed batch of the systems module
    ref = systems.batched_rocksalt(256, seed=bench.SEED)
    assert bench.workload_config(256, 1)["particles_per_gpu"] == sum(s.N for s in ref)


def test_water_row_filter():
    assert bench.water_rows("") == set()
    assert bench.water_rows("1e-5:f64, 1e-3:f32") == {(1e-5, "f64"), (1e-3, "f32")}
    with pytest.raises(ValueError):
        bench.water_rows("1e-5:f16")
