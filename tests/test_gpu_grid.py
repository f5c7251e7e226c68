"""GPU construction of the grid cell lists (qmcrt_grid_build_device, csrc/grid_build.cu)
against the host's lists (csrc/scene.cpp match_grid, the restatement of the
reference's RectangleGrid::CGridHelioMatch, which tests/test_oracle_golden.py
pins to the reference's own outputs).

Bar (written here): the device-built ranges and entries equal the host's
entry for entry (integer lists: bit-exact), on a flat field, a focus-flat
field, an uneven field of the batch benchmark, a two-grid scene and the
10,000-heliostat field; a trace after the rebuild equals one before.
"""
import time

import numpy as np
import pytest

import solarenergy_chier_b200 as q
from solarenergy_chier_b200 import synth

pytestmark = pytest.mark.gpu


def fields(kind, tmp_path):
    if kind == "small":
        return synth.small_field(tmp_path, seed=2, helio_pixel=0.5)
    if kind == "large":
        return synth.large_field(tmp_path, seed=4, num_heliostats=200, helio_pixel=0.25, receiver_pixel=0.05,
                                 groups=4, per_group=128)
    if kind == "uneven":
        return synth.uneven_field(tmp_path, 5, seed=0, helio_pixel=1.0, groups=4, per_group=128)
    if kind == "two":
        return synth.two_receiver_field(tmp_path, seed=1)
    return synth.huge_field(tmp_path, seed=0, helio_pixel=1.0, groups=4, per_group=128)


@pytest.mark.parametrize("kind", ["small", "large", "uneven", "two", "huge"])
def test_device_grid_build_equals_host(kind, tmp_path, cuda_device):
    f = fields(kind, tmp_path)
    t0 = time.perf_counter()
    q.Scene(f.scene, f.config, device=-1).close()
    host_load_s = time.perf_counter() - t0
    s = q.Scene(f.scene, f.config, device=0, seed=3)
    s.set_math_mode(1)
    s.set_light_range(0, 16)
    ids = list(range(s.num_heliostats))
    s.trace(ids)
    before = s.power()[0]
    for g in range(s.num_grids):
        r0, e0 = s.device_grid_cells(g)
        ms = s.build_grid_on_device(g)
        r1, e1 = s.device_grid_cells(g)
        assert np.array_equal(r0, r1), f"grid {g}: cell ranges differ"
        assert np.array_equal(e0, e1), f"grid {g}: cell entries differ"
        assert e0.shape[0] > 0
        print(f"{kind} grid {g}: {s.num_heliostats} heliostats, {r0.shape[0]} cells, {e0.shape[0]} entries, "
              f"device build {ms:.3f} ms (host-only scene load incl. parsing {1e3 * host_load_s:.1f} ms)")
    s.clear()
    s.clear_power()
    s.trace(ids)
    np.testing.assert_allclose(s.power()[0], before, rtol=1e-12, atol=0)
