"""The CPU oracle against the reference's own known answers and golden outputs.

Two kinds of pins:
  * the expectations written in the reference's gtest suites
    (Tests/DataStructureTests/*, Tests/QuasiMonteCarloRayTracingTests/*),
    restated here as literals, at the tolerances those tests use;
  * tests/golden/*.npz, outputs of the reference's own host code
    (tests/golden/make_golden.py), compared exactly.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle, scene_text
from tests.conftest import GOLDEN
from tests.golden.fixtures import offsets_for


def close3(a, b, tol):
    return np.all(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)) < tol)


# ---- Tests/DataStructureTests/CylinderReceiverTest.cpp ------------------------
POS0 = [0.0, 0.0, 0.0]
SIZE0 = [3.0, 4.0, 0.0]


def norm(v):
    v = np.asarray(v, np.float32)
    return (v / np.sqrt(np.dot(v, v))).astype(np.float32)


def test_cylinder_resolution():
    # CylinderReceiverTest.cpp:25-29
    assert oracle.probe_cylinder_resolution(SIZE0, 3) == (57, 12)


@pytest.mark.parametrize("origin,direction,expect", [
    ((1.5, 0.0, -6.0), (0.0, 0.0, 1.0), (6 - 1.5 * math.sqrt(3), 0.5, 5.0 / 6.0)),
    ((1.5, 0.0, -6.0), tuple(norm([-1.0, 0.0, 2.0])), (1.5 * math.sqrt(5), 0.5, 0.75)),
    ((1.5, 2.0, -6.0), tuple(norm([-1.0, 0.0, 2.0])), (1.5 * math.sqrt(5), 1.0, 0.75)),
    ((-6.0, 0.0, -1.5), (1.0, 0.0, 0.0), (6 - 1.5 * math.sqrt(3), 0.5, 7.0 / 12.0)),
    ((3.0, 0.0, 3.0), (-1.0, 0.0, 0.0), (3.0, 0.5, 0.25)),
])
def test_cylinder_has_intersection(origin, direction, expect):
    # CylinderReceiverTest.cpp:32-64 (1e-4, all three components checked)
    hit, tuv = oracle.probe_cylinder_hit(POS0, SIZE0, origin, direction)
    assert hit
    assert close3(tuv, expect, 1e-4)


def test_cylinder_boundary_intersection():
    # CylinderReceiverTest.cpp:67-76
    hit, _ = oracle.probe_cylinder_hit([0.0, 0.0, -3.0], [3.0, 8.0, 0.0], [-7.673, -0.575, -3.224],
                                       norm([0.999, 0.010, 0.048]))
    assert hit


@pytest.mark.parametrize("origin,direction", [
    ((1.0, 1.0, 1.0), (1.0, 0.0, 0.0)),
    ((0.0, -2.1, -5.0), (0.0, 0.0, 1.0)),
    ((1.0, 2.5, -3.0), tuple(norm([-0.1, 0.0, 1.0]))),
])
def test_cylinder_no_intersection(origin, direction):
    # CylinderReceiverTest.cpp:78-96
    hit, _ = oracle.probe_cylinder_hit(POS0, SIZE0, origin, direction)
    assert not hit


def test_cylinder_focus_centres():
    # CylinderReceiverTest.cpp:98-137
    pos, r = [2.0, 3.0, 1.0], 3.0
    s2 = r * math.sqrt(2) / 2
    assert close3(oracle.probe_cylinder_focus(pos, SIZE0, [5, 0, -2]), [s2 + 2, 3, 1 - s2], 1e-4)
    assert close3(oracle.probe_cylinder_focus(pos, SIZE0, [8, 4, 1]), [5, 3, 1], 1e-4)
    d = np.array([6.0, -1.0]) / math.hypot(6.0, -1.0)
    dist = math.hypot(-4 - 2, 2 - 1) - r
    exp = [-4 + dist * d[0], 3, 2 + dist * d[1]]
    assert close3(oracle.probe_cylinder_focus(pos, SIZE0, [-4, 6, 2]), exp, 1e-4)
    exp[2] = 2 - exp[2]
    assert close3(oracle.probe_cylinder_focus(pos, SIZE0, [-4, 1, 0]), exp, 1e-4)
    assert close3(oracle.probe_cylinder_focus(POS0, SIZE0, [0, 0, -6]), [0, 0, -3], 1e-4)
    assert close3(oracle.probe_cylinder_focus(POS0, SIZE0, [3, 0, -3]), [3 / math.sqrt(2), 0, -3 / math.sqrt(2)], 1e-4)
    assert close3(oracle.probe_cylinder_focus(POS0, SIZE0, [1, 1, 1]), POS0, 1e-4)


# ---- Tests/DataStructureTests/RectangleGridTest.cpp ----------------------------
GRID_HELIOS = [((-8, 5, 25), 1.5), ((10, 5, 22.5), 0.75), ((10, 5, 27.5), 0.75), ((-10, 5, 35), 1.0),
               ((0, 5, 35), 1.0)]


def _grid(nsub):
    hp = np.array([p for p, _ in GRID_HELIOS], np.float32)
    hs = np.array([np.array([4.0, 0.1, 3.0], np.float32) * np.float32(k) for _, k in GRID_HELIOS], np.float32)
    return oracle.probe_grid([-15, 0, 20], [30, 10, 20], [10, 10, 10], hp, hs, nsub)


def test_grid_cell_lists_one_subheliostat():
    # RectangleGridTest.cpp:83-117
    index, match = _grid([1, 1, 1, 1, 1])
    assert index.tolist() == [0, 1, 2, 3, 4, 6, 6]
    assert match.tolist() == [0, 3, 0, 4, 1, 2]


def test_grid_cell_lists_many_subheliostats():
    # RectangleGridTest.cpp:120-159
    index, match = _grid([1, 2, 3, 4, 5])
    assert index.tolist() == [0, 1, 5, 6, 11, 16, 16]
    assert match.tolist() == [0, 6, 7, 8, 9, 0, 10, 11, 12, 13, 14, 1, 2, 3, 4, 5]


# ---- Tests/DataStructureTests/RectangleHelioTest.cpp ---------------------------
def test_flat_heliostat_microfacets():
    # RectangleHelioTest.cpp:48-94 (1e-3)
    h = oracle.probe_heliostat(0, [6.0, 0.1, 5.0], [2.0, 1.0], [3, 2], 1.0, [0, 1, 0], [0, 0, 0])
    expect = [(-2.5, 0.05, -2.0), (-1.5, 0.05, -2.0), (1.5, 0.05, -2.0), (2.5, 0.05, -2.0),
              (-2.5, 0.05, 0.0), (-1.5, 0.05, 0.0), (1.5, 0.05, 0.0), (2.5, 0.05, 0.0),
              (-2.5, 0.05, 2.0), (-1.5, 0.05, 2.0), (1.5, 0.05, 2.0), (2.5, 0.05, 2.0)]
    assert h["origins"].shape == (12, 3)
    assert close3(h["origins"], expect, 1e-3)
    assert close3(h["normals"], [(0, 1, 0)] * 12, 1e-3)


# ---- Tests/DataStructureTests/FocusFlatRectangleHelioTest.cpp ------------------
FF_NORMALS = [norm(v) for v in ([0.3, 1.0, 0.325], [0.0, 1.0, 0.325], [-0.3, 1.0, 0.325], [0.3, 1.0, -0.325],
                                [0.0, 1.0, -0.325], [-0.3, 1.0, -0.325])]
FF_CENTRES = [(-0.6, 0.245625, -0.65), (0.0, 0.155625, -0.65), (0.6, 0.245625, -0.65), (-0.6, 0.245625, 0.65),
              (0.0, 0.155625, 0.65), (0.6, 0.245625, 0.65)]
FF_POS = np.array([10.0, 2.0, 6.0])


def _ff():
    return oracle.probe_heliostat(1, [1.7, 0.1, 2.3], [0.1, 0.3], [2, 3], 0.5, [0, 1, 0], FF_POS, focus_length=1.0)


def _local2world(d, n):
    # global_func::local2world_rotate (Util/global_function.cuh:19-36) in float64
    d, n = np.asarray(d, np.float64), np.asarray(n, np.float64)
    if abs(n[0]) < 1e-5 and abs(n[2]) < 1e-5:
        return d
    u = np.cross([0.0, 1.0, 0.0], n)
    u /= np.linalg.norm(u)
    v = np.cross(u, n)
    v /= np.linalg.norm(v)
    return d[0] * u + d[1] * n + d[2] * v


def _transfer(p, ln, lc):
    # microHeliostatPointLocalTransfer, heliostat normal (0,1,0)
    return _local2world(p, ln) + np.asarray(lc)


def test_focus_flat_local_frames():
    # FocusFlatRectangleHelioTest.cpp:120-130
    h = _ff()
    assert close3(h["local_centers"], FF_CENTRES, 1e-3)
    assert close3(h["local_normals"], FF_NORMALS, 1e-3)


def test_focus_flat_subheliostat_vertices():
    # FocusFlatRectangleHelioTest.cpp:136-202
    lb, lu, ru, rb = (-0.25, 0.0, 0.5), (-0.25, 0.0, -0.5), (0.25, 0.0, -0.5), (0.25, 0.0, 0.5)
    t00 = {k: _transfer(v, FF_NORMALS[0], FF_CENTRES[0]) for k, v in dict(lb=lb, lu=lu, ru=ru, rb=rb).items()}
    t01 = {k: _transfer(v, FF_NORMALS[1], FF_CENTRES[1]) for k, v in dict(lb=lb, lu=lu, ru=ru, rb=rb).items()}
    nx = lambda v: np.array([-v[0], v[1], v[2]])  # noqa: E731
    nz = lambda v: np.array([v[0], v[1], -v[2]])  # noqa: E731
    expect = [t00["lb"], t00["lu"], t00["ru"], t01["lb"], t01["lu"], t01["ru"],
              nx(t00["rb"]), nx(t00["ru"]), nx(t00["lu"]),
              nz(t00["lu"]), nz(t00["lb"]), nz(t00["rb"]), nz(t01["lu"]), nz(t01["lb"]), nz(t01["rb"]),
              nx(nz(t00["ru"])), nx(nz(t00["rb"])), nx(nz(t00["lb"]))]
    expect = np.array(expect) + FF_POS
    assert close3(_ff()["subverts"], expect, 1e-3)


def test_focus_flat_microfacets():
    # FocusFlatRectangleHelioTest.cpp:208-288
    up, bottom = (0.0, 0.0, -0.25), (0.0, 0.0, 0.25)
    p00 = _transfer(up, FF_NORMALS[0], FF_CENTRES[0])
    p10 = _transfer(bottom, FF_NORMALS[0], FF_CENTRES[0])
    p01 = _transfer(up, FF_NORMALS[1], FF_CENTRES[1])
    p11 = _transfer(bottom, FF_NORMALS[1], FF_CENTRES[1])
    nx = lambda v: np.array([-v[0], v[1], v[2]])  # noqa: E731
    nz = lambda v: np.array([v[0], v[1], -v[2]])  # noqa: E731
    expect = np.array([p00, p01, nx(p00), p10, p11, nx(p10), nz(p10), nz(p11), nx(nz(p10)), nz(p00), nz(p01),
                       nx(nz(p00))]) + FF_POS
    nrm = [FF_NORMALS[i] for i in (0, 1, 2, 0, 1, 2, 3, 4, 5, 3, 4, 5)]
    h = _ff()
    assert close3(h["origins"], expect, 1e-3)
    assert close3(h["normals"], nrm, 1e-3)


# ---- Tests/QuasiMonteCarloRayTracingTests/QuasiMonteCarloRayTracerTest.cpp -----
def test_tracer_vertex_table_and_facets(reference_tests_scene):
    o = reference_tests_scene
    g = o.grid(0)
    v = g["vertices"]
    # QuasiMonteCarloRayTracerTest.cpp:110-124: heliostat 1 and 3 (the test swaps
    # heliostat 2 for a fake type), tolerance 1e-2
    assert close3(v[0:3], [(2.0, 1.5, 7.85), (2.0, -1.5, 7.85), (-2.0, -1.5, 7.85)], 1e-2)
    assert close3(v[6:9], [(-3.40423, 2.09987, 20.1253), (-3.40541, -1.90012, 20.135), (-6.38378, -1.90012, 19.7754)],
                  1e-2)
    # :127-144 heliostat 0 micro-facets, normals (0, 0, -1)
    origins, normals = o.facets(0)
    expect = [(1.5, 1.0, 7.85), (0.5, 1.0, 7.85), (-0.5, 1.0, 7.85), (-1.5, 1.0, 7.85), (1.5, 0.0, 7.85),
              (0.5, 0.0, 7.85), (-0.5, 0.0, 7.85), (-1.5, 0.0, 7.85), (1.5, -1.0, 7.85), (0.5, -1.0, 7.85),
              (-0.5, -1.0, 7.85), (-1.5, -1.0, 7.85)]
    assert close3(origins, expect, 1e-3)
    assert close3(normals, [(0, 0, -1)] * 12, 1e-3)


def test_subheliostat_ids_are_prefix_sums():
    # QuasiMonteCarloRayTracerTest.cpp:159-162 (subHeliostat_id = sub-heliostats before it in its grid)
    sc = scene_text.parse_scene((GOLDEN / "synth_small_scene.scn").read_text())
    cfg, _ = scene_text.parse_config((GOLDEN / "synth_small_configuration.json").read_text())
    o = oracle.OracleScene(sc, cfg)
    assert [o.heliostat(i)["sub_begin"] for i in range(5)] == [0, 1, 2, 3, 4]


@pytest.fixture(scope="module")
def reference_tests_scene():
    scn = """# Tests/QuasiMonteCarloRayTracingTests/test_file/test_scene.scn, restated
ground 1024.000000 1024.000000
ngrid 1
Recv 0
pos 0.000000 0.000000 -1.50000
size 16.000000 10.000000 3.000000
norm 0.000000 0.000000 1.000000
face 0
end
Grid 0
pos -15.00000 -4.500000 0.0000000
size 20.000000 9.0000000 24.000000
inter 10.000000 9.0000000 8.0000000
n 3
type 0
end
helio 0.0000000 0.0000000 7.9000000
4.0000000 0.1000000 3.0000000
gap 1.0000000 0.5000000
matrix 3 2
helio 0.0000000 0.0000000 12.000000
5.0000000 0.1000000 4.0000000
matrix 1 1
helio -4.900000 0.1000000 20.000000
3.0000000 0.1000000 4.0000000
"""
    cfg = {"sun_dir": [0.0, 0.0, 1.0], "csr": 0.1, "dni": 500.0, "num_of_sunshape_groups": 32,
           "num_per_sunshape_group": 2048, "inverse_transform_sampling_groups": 64, "receiver_pixel_length": 0.5,
           "helio_disturb_std": 0.02, "helio_reflected_rate": 2.0, "helio_pixel_length": 1.0}
    c, _ = scene_text.parse_config(json.dumps(cfg))
    return oracle.OracleScene(scene_text.parse_scene(scn), c)


# ---- golden outputs of the reference's own code (tests/golden/) -----------------
GOLDEN_CASES = sorted(p.stem.split("_", 1)[1] for p in GOLDEN.glob("geometry_*.npz"))


def _case_files(name):
    """Scene and configuration of a golden case, from the reference tree when
    present, else from the restated copies kept next to the fixtures."""
    from tests.golden import make_golden as mg

    if name == "synth_small":
        return GOLDEN / "synth_small_scene.scn", GOLDEN / "synth_small_configuration.json"
    scn, cfg = mg.CASES[name]
    return mg.REF / scn, mg.REF / cfg


def _oracle_for(name, trace_cfg=False):
    scn, cfg = _case_files(name)
    if not Path(scn).exists():
        pytest.skip("reference scene file not available on this machine")
    if trace_cfg and name != "synth_small":
        cfg = GOLDEN / f"cfg_{name}.json"
    return oracle.OracleScene.from_files(scn, cfg)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_geometry(name):
    g = np.load(GOLDEN / f"geometry_{name}.npz")
    o = _oracle_for(name)
    assert [o.num_receivers, o.num_grids, o.num_heliostats] == g["counts"].tolist()
    for i in range(o.num_receivers):
        r = o.receiver(i)
        assert [r["type"], r["width"], r["height"]] == g[f"recv{i}_size"].tolist()
        assert np.array_equal(r["vertices"].astype(np.float32), g[f"recv{i}_vertices"])
    for k in range(o.num_grids):
        gd = o.grid(k)
        assert list(gd["cells"]) == g[f"grid{k}_cells"].tolist()
        assert np.array_equal(gd["index"], g[f"grid{k}_index"])
        assert np.array_equal(gd["match"], g[f"grid{k}_match"])
        assert np.array_equal(gd["vertices"].astype(np.float32), g[f"grid{k}_vertices"])
    ints = np.array([[o.heliostat(h)[k] for k in ("type", "grid", "num_facets", "num_sub", "sub_begin")]
                     for h in range(o.num_heliostats)])
    assert np.array_equal(ints, g["helio_ints"])
    normals = np.array([o.heliostat(h)["normal"] for h in range(o.num_heliostats)], np.float32)
    assert np.array_equal(normals, g["helio_normals"])
    for h in range(min(o.num_heliostats, 3)):
        origins, fn = o.facets(h)
        idx = g[f"facets{h}_index"]
        assert np.array_equal(origins[idx].astype(np.float32), g[f"facets{h}_origins"])
        assert np.array_equal(fn[idx].astype(np.float32), g[f"facets{h}_normals"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_trace(name):
    t = np.load(GOLDEN / f"trace_{name}.npz")
    o = _oracle_for(name, trace_cfg=True)
    P = o.pool_size
    nf = [o.heliostat(h)["num_facets"] for h in range(o.num_heliostats)]
    offs = offsets_for(nf, P, int(t["offset_seed"]))
    lights = int(t["lights"])
    for h in t["ids"].tolist():
        fe = min(nf[h], 256)
        res = o.trace([h], t["pool_dirs"], t["pool_pert"], offs, 0, lights, record=(h, 0, fe))
        assert np.array_equal(res["records"], t[f"records{h}"]), "per-ray outcome differs from the reference"
        assert res["power"][h] == float(t[f"power{h}"])
        for k, img in enumerate(res["images"]):
            flat = img.ravel()
            idx = t[f"image{h}_{k}_index"]
            assert np.array_equal(np.nonzero(flat)[0], idx)
            assert np.array_equal(flat[idx], t[f"image{h}_{k}_value"])
        c = res["counters"]
        assert [c[k] for k in ("rays", "shadowed", "blocked", "missed", "hit", "clamped")] == t[f"counters{h}"].tolist()


def test_golden_smoother():
    s = np.load(GOLDEN / "smooth.npz")
    k = 0
    while f"in{k}" in s:
        rad, ratio = s[f"params{k}"]
        out = oracle.smooth(s[f"in{k}"], int(rad), float(ratio))
        assert np.array_equal(out, s[f"out{k}"]), f"smoother case {k}"
        k += 1
    assert k >= 4


def test_golden_buie():
    b = np.load(GOLDEN / "buie.npz")
    k = 0
    while f"u{k}" in b:
        csr, groups = b[f"params{k}"]
        t = oracle.buie_table(float(csr), int(groups))
        for key in ("cdf_x", "cdf_y", "k"):
            assert np.array_equal(t[key], b[f"{key}{k}"])
        for key in ("less_465", "gamma", "A", "B", "C"):
            assert np.float32(t[key]) == np.float32(b[f"{key}{k}"])
        theta = oracle.buie_theta(float(csr), int(groups), b[f"u{k}"])
        assert np.array_equal(theta, b[f"theta{k}"])
        k += 1
    assert k >= 3
