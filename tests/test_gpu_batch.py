"""Batched tracing (qmcrt_batch_*) against the plain path, on the GPU.

A batch instance (scene, sun) must behave exactly like the plain scene after
qmcrt_scene_set_sun(sun): the device-prepared geometry is bit-identical to
the host's, and in the exact math mode per-ray outcomes are identical, so
flux images agree up to the order of float atomic accumulation
(L1 <= 1e-5) and FP64 powers up to summation order (<= 1e-9 relative).
"""
import numpy as np
import pytest

import solarenergy_chier_b200 as q
from solarenergy_chier_b200 import synth

pytestmark = pytest.mark.gpu

SUNS = [[0.0, -0.866, -0.5], [0.35, -0.75, 0.56], [-0.5, -0.6, 0.62]]


@pytest.fixture(scope="module")
def fields(tmp_path_factory, cuda_device):
    big = synth.large_field(tmp_path_factory.mktemp("b1"), seed=6, num_heliostats=24, helio_pixel=0.25,
                            receiver_pixel=0.05, groups=4, per_group=128)
    small = synth.small_field(tmp_path_factory.mktemp("b2"), seed=2, helio_pixel=0.2, groups=4, per_group=128)
    return big, small


def scenes_of(fields):
    return [q.Scene(f.scene, f.config, device=0, seed=11) for f in fields]


def plain_reference(f, sun, mode):
    s = q.Scene(f.scene, f.config, device=0, seed=11)
    s.set_sun(sun)
    s.set_math_mode(mode)
    s.trace(list(range(s.num_heliostats)))
    per, total = s.power()
    return s, s.image(0), per, total


def test_device_preparation_equals_host(fields):
    scenes = scenes_of(fields)
    inst = [(0, SUNS[0]), (0, SUNS[1]), (1, SUNS[2]), (1, SUNS[0])]
    b = q.Batch(scenes, inst)
    for k, (si, sun) in enumerate(inst):
        ref = q.Scene(fields[si].scene, fields[si].config, device=-1)
        ref.set_sun(sun)
        verts, normals = b.geometry(k, 0)
        assert np.array_equal(verts, ref.grid(0)["vertices"]), f"instance {k}: vertices differ"
        want = np.stack([ref.heliostat(h)["normal"] for h in range(ref.num_heliostats)])
        assert np.array_equal(normals, want), f"instance {k}: normals differ"


@pytest.mark.parametrize("mode", [1, 0])
def test_batch_equals_plain_per_sun(fields, mode):
    scenes = scenes_of(fields)
    inst = [(0, SUNS[0]), (0, SUNS[1]), (1, SUNS[2]), (1, SUNS[1])]
    b = q.Batch(scenes, inst)
    b.set_math_mode(mode)
    b.trace()
    for k, (si, sun) in enumerate(inst):
        _, img, per, total = plain_reference(fields[si], sun, mode)
        got = b.image(k).astype(np.float64)
        l1 = np.abs(got - img).sum() / img.sum()
        assert l1 <= 1e-5, f"instance {k}: flux L1 {l1:.2e}"
        gper, gtotal = b.power(k)
        assert abs(gtotal - total) <= 1e-9 * total
        assert np.allclose(gper, per, rtol=1e-9, atol=0)


def test_graph_replay_and_set_suns(fields):
    scenes = scenes_of(fields)
    inst = [(0, SUNS[0]), (1, SUNS[1])]
    b = q.Batch(scenes, inst)
    b.set_math_mode(1)
    b.set_light_range(0, 64)
    b.trace()
    first = [b.image(k) for k in range(2)]
    b.capture_graph(clear_first=True)
    b.graph_launch()
    b.graph_launch()  # clears, then traces again: same images
    for k in range(2):
        assert np.abs(b.image(k) - first[k]).sum() <= 1e-5 * first[k].sum()
    # new suns prepared on the device equal a plain scene with those suns
    b.set_suns([SUNS[2], SUNS[0]])
    b.clear()
    b.set_light_range(0, 128)
    b.trace()
    for k, (si, sun) in enumerate([(0, SUNS[2]), (1, SUNS[0])]):
        _, img, _, total = plain_reference(fields[si], sun, 1)
        assert np.abs(b.image(k) - img).sum() <= 1e-5 * img.sum()
        assert abs(b.power(k)[1] - total) <= 1e-9 * total


def test_autotune_and_errors(fields):
    scenes = scenes_of(fields)
    b = q.Batch(scenes, [(0, SUNS[0]), (1, SUNS[1])])
    shape, ms = b.autotune()
    assert 0 <= shape < len(q.launch_shapes()) and len(ms) == len(q.launch_shapes()) and min(ms) > 0
    assert ms[shape] == min(ms)
    assert b.power(0)[1] == 0.0  # autotune clears
    with pytest.raises(q.QmcrtError):
        b.set_light_range(0, 10 ** 6)
    with pytest.raises(q.QmcrtError):
        b.image(5)
    with pytest.raises(q.QmcrtError):
        b.graph_launch()
    with pytest.raises(q.QmcrtError):
        q.Batch(scenes, [(2, SUNS[0])])
    with pytest.raises(q.QmcrtError):
        q.Batch(scenes, [(0, [0.0, 0.0, 0.0])])


def test_uneven_fields_batch_equals_plain(tmp_path):
    """Two of the batch benchmark's uneven fields (a rectangle receiver with
    flat heliostats, a cylinder with focus-flat ones), coarse facets, at
    their own suns and at a shared one, in one batch with mismatched sizes."""
    files = [synth.uneven_field(tmp_path, k, seed=3, helio_pixel=0.75, groups=4, per_group=128) for k in (0, 1)]
    scenes = [q.Scene(f.scene, f.config, device=0, seed=11) for f in files]
    own = [np.array(s.info.sun_dir[:], np.float32) for s in scenes]
    inst = [(0, own[0]), (1, own[1]), (1, SUNS[1]), (0, SUNS[2])]
    b = q.Batch(scenes, inst)
    b.set_math_mode(1)
    b.trace()
    for k, (si, sun) in enumerate(inst):
        _, img, per, total = plain_reference(files[si], sun, 1)
        assert total > 0, f"instance {k}: no energy"
        got = b.image(k).astype(np.float64)
        assert np.abs(got - img).sum() <= 1e-5 * img.sum(), f"instance {k}"
        gper, gtotal = b.power(k)
        assert abs(gtotal - total) <= 1e-9 * total
        assert np.allclose(gper, per, rtol=1e-9, atol=0)


def test_every_launch_shape_gives_the_same_result(fields, tmp_path):
    """The autotuner's candidates (launch shapes of the production build:
    block widths, warp chunks of 32, 64 or 128 iterations) change only how
    rays are handed to warps: every shape gives the same flux (up to float
    atomic order, L1 <= 1e-6) and FP64 powers (1e-12) on a plain scene and
    on a batch, with ragged light counts (37 lights: warps span facets and
    chunks end inside one), and the plain autotuner keeps the fastest."""
    shapes = q.launch_shapes()
    assert shapes[0] == (32, 64, False) and len(shapes) >= 5 and any(x[2] for x in shapes)
    f = fields[1]
    s = q.Scene(f.scene, f.config, device=0, seed=4)
    ids = list(range(s.num_heliostats))
    s.set_light_range(3, 40)
    ref = None
    for k in range(len(shapes)):
        s.set_launch_shape(k)
        s.clear()
        s.clear_power()
        s.trace(ids)
        img = s.image(0).astype(np.float64)
        per, total = s.power()
        if ref is None:
            ref = (img, per, total)
            assert total > 0
            continue
        assert np.abs(img - ref[0]).sum() <= 1e-6 * ref[0].sum(), shapes[k]
        np.testing.assert_allclose(per, ref[1], rtol=1e-12, atol=0)
    best, ms = s.autotune(ids)
    assert ms[best] == min(ms) and min(ms) > 0
    assert s.power()[1] == 0.0
    s.trace(ids)  # the chosen shape traces like the others
    assert abs(s.power()[1] - ref[2]) <= 1e-12 * ref[2]
    scenes = scenes_of(fields)
    b = q.Batch(scenes, [(0, SUNS[0]), (1, SUNS[1])])
    b.set_light_range(1, 38)
    first = None
    for k in range(len(shapes)):
        b.set_launch_shape(k)
        b.clear()
        b.trace()
        out = [(b.image(i).astype(np.float64), b.power(i)[1]) for i in range(2)]
        if first is None:
            first = out
            continue
        for (img, tot), (img0, tot0) in zip(out, first):
            assert np.abs(img - img0).sum() <= 1e-6 * img0.sum()
            assert abs(tot - tot0) <= 1e-12 * tot0
