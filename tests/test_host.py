"""Host-side logic of the product, on CPU: scene/configuration/task readers,
float32 scene geometry, flux-map text output and the C ABI's exports.

The product's geometry is compared bit for bit with the CPU oracle; the
readers' accept/reject decisions follow the reference's own tests
(Tests/DataStructureTests/SceneLoaderTest.cpp, SceneConfigurationTest.cpp,
Tests/RayTracingPipelineTests/TaskLoaderTest.cpp).
"""
import ctypes
import json
import os
import re
from pathlib import Path

import numpy as np
import pytest

import solarenergy_chier_b200 as q
from oracle import oracle, scene_text
from solarenergy_chier_b200 import synth
from tests.conftest import GOLDEN, ROOT

REF = Path(os.environ.get("QMCRT_REFERENCE_TREE", "/root/reference"))
GOOD_SCENE = """# Tests/DataStructureTests/test_file/test_scene_good.scn, restated
ground 1024.000000 1024.000000
ngrid 2
Recv 0
pos 0.000000 100.000000 0.000000
size 16.000000 10.000000 3.000000
norm 0.000000 0.000000 1.000000
face 0
end
Grid 0
pos -14.00000 5.0000000 -56.00000
size 28.000000 14.000000 28.000000
inter 14.000000 14.000000 14.000000
n 4
type 0
end
gap 0.100000 0.200000
matrix 2 2
helio -7.000000 12.000000 -35.00000
10.000000 0.1000000 8.0000000
gap 1.000000 1.00000
helio -7.000000 12.000000 -49.00000
10.000000 0.1000000 8.0000000
matrix 4 2
helio 7.0000000 12.000000 -35.00000
10.000000 0.1000000 8.0000000
helio 7.0000000 12.000000 -49.00000
10.000000 0.1000000 8.0000000
Grid 0
pos -14.00000 5.0000000 28.000000
size 28.000000 14.000000 28.000000
inter 14.000000 14.000000 14.000000
n 4
type 0
end
gap 0.100000 0.100000
matrix 2 2
helio -7.000000 12.000000 35.000000
10.000000 0.1000000 8.0000000
helio -7.000000 12.000000 49.000000
10.000000 0.1000000 8.0000000
helio 7.0000000 12.000000 35.000000
10.000000 0.1000000 8.0000000
helio 7.0000000 12.000000 49.000000
10.000000 0.1000000 8.0000000
"""
CONFIG = {"sun_dir": [0.0, -1.0, 0.0], "csr": 0.1, "dni": 500.0, "num_of_sunshape_groups": 32,
          "num_per_sunshape_group": 2048, "inverse_transform_sampling_groups": 64, "receiver_pixel_length": 0.05,
          "helio_disturb_std": 0.02, "helio_reflected_rate": 2.0, "helio_pixel_length": 0.10}


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return p


def load_host(scn, cfg):
    return q.Scene(scn, cfg, device=-1)


def assert_same_geometry(p: q.Scene, o: oracle.OracleScene):
    assert (p.num_receivers, p.num_grids, p.num_heliostats) == (o.num_receivers, o.num_grids, o.num_heliostats)
    for i in range(p.num_receivers):
        a, b = p.receiver(i), o.receiver(i)
        assert (a["type"], a["width"], a["height"]) == (b["type"], b["width"], b["height"])
        assert np.array_equal(a["vertices"].astype(np.float64), b["vertices"])
        assert a["pixel_length"] == np.float32(b["pixel_length"])
    for g in range(p.num_grids):
        a, b = p.grid(g), o.grid(g)
        assert a["cells"] == b["cells"]
        assert np.array_equal(a["index"], b["index"]) and np.array_equal(a["match"], b["match"])
        assert np.array_equal(a["vertices"].astype(np.float64), b["vertices"])
    for h in range(p.num_heliostats):
        a, b = p.heliostat(h), o.heliostat(h)
        for k in ("type", "grid", "num_facets", "num_sub", "sub_begin"):
            assert a[k] == b[k], k
        assert np.array_equal(a["normal"].astype(np.float64), b["normal"])


# ---- readers ----------------------------------------------------------------
def test_good_scene_loads(tmp_path):
    cfg = write(tmp_path, "c.json", json.dumps(CONFIG))
    s = load_host(write(tmp_path, "good.scn", GOOD_SCENE), cfg)
    assert (s.num_receivers, s.num_grids, s.num_heliostats) == (1, 2, 8)
    # matrix 4x2 on a flat heliostat changes its facets, not its sub-heliostat count
    assert s.heliostat(2)["num_sub"] == 1
    assert s.heliostat(2)["num_facets"] == 4 * 2 * int((8.0 - 1.0 * 3) / 4 / 0.1) * int((10.0 - 1.0) / 2 / 0.1)


@pytest.mark.parametrize("mutate,why", [
    (lambda t: t.replace("ngrid 2", "ngrid 3"), "grid count"),                        # bad_corresponding
    (lambda t: t.replace("n 4\ntype 0\nend\ngap 0.100000 0.200000", "n 5\ntype 0\nend\ngap 0.100000 0.200000"),
     "heliostat count"),                                                              # bad_corresponding2
    (lambda t: t.replace("Grid 0\npos -14.00000 5.0000000 -56", "test 0\npos -14.00000 5.0000000 -56"),
     "unknown field"),                                                                # bad_unknownFields
    (lambda t: t.replace("end\nGrid 0\npos -14.00000 5.0000000 -56",
                         "end\nRecv 0\npos 0 100 0\nsize 16 10 3\nnorm 0 0 1\nface 0\nend\nGrid 0\npos -14.00000 5.0000000 -56"),
     "grammar"),                                                                      # bad_nonRE
    (lambda t: t.replace("inter 14.000000 14.000000 14.000000\nn 4", "interval 14 14 14\nn 4", 1), "missing key"),
    (lambda t: t.replace("Recv 0", "Recv 7"), "receiver type"),
    (lambda t: t.replace("type 0\nend\ngap 0.100000 0.200000", "type 9\nend\ngap 0.100000 0.200000"),
     "heliostat type"),
])
def test_bad_scenes_are_rejected(tmp_path, mutate, why):
    cfg = write(tmp_path, "c.json", json.dumps(CONFIG))
    bad = write(tmp_path, "bad.scn", mutate(GOOD_SCENE))
    with pytest.raises(q.QmcrtError) as e:
        load_host(bad, cfg)
    assert e.value.code == 2, why
    with pytest.raises(scene_text.SceneError):
        scene_text.parse_scene(bad.read_text())


def test_reference_scene_files_agree_with_reference_loader():
    from oracle import refhost

    if not refhost.available():
        pytest.skip("reference host library not built")
    folder = REF / "Tests/DataStructureTests/test_file"
    if not folder.exists():
        pytest.skip("reference tree not mounted")
    cfg = folder / "test_configuration.json"
    for scn in sorted(folder.glob("*.scn")):
        ref_ok = refhost.read_scene(scn)
        try:
            load_host(scn, cfg)
            ok = True
        except q.QmcrtError:
            ok = False
        assert ok == ref_ok, scn.name


def test_config_field_counts(tmp_path):
    # SceneConfigurationTest.cpp:32-68: 10 fields, 8 fields, malformed -> throw, missing -> throw
    full = write(tmp_path, "full.json", json.dumps(CONFIG))
    part = dict(CONFIG)
    del part["sun_dir"], part["inverse_transform_sampling_groups"]
    partial = write(tmp_path, "partial.json", json.dumps(part))
    scn = write(tmp_path, "good.scn", GOOD_SCENE)
    assert load_host(scn, full).info.config_fields == 10
    s = load_host(scn, partial)
    assert s.info.config_fields == 8
    assert list(s.info.sun_dir) == [1.0, 0.0, 0.0]          # default kept
    assert s.info.inverse_transform_sampling_groups == 1024
    invalid = write(tmp_path, "invalid.json", '{\n "csr": 1.0,\n "dni": 500.0,\n AGG\n}')
    with pytest.raises(q.QmcrtError):
        load_host(scn, invalid)
    with pytest.raises(q.QmcrtError):
        load_host(scn, tmp_path / "missing.json")


def test_config_values_round_like_the_reference(tmp_path):
    cfg = dict(CONFIG, receiver_pixel_length=0.02, helio_pixel_length=0.0123456789, dni=987.654321)
    path = write(tmp_path, "c.json", json.dumps(cfg))
    s = load_host(write(tmp_path, "good.scn", GOOD_SCENE), path)
    parsed, n = scene_text.parse_config(path.read_text())
    assert n == 10
    assert np.float32(s.info.helio_pixel_length) == parsed["helio_pixel_length"]
    assert np.float32(s.info.dni) == parsed["dni"]


@pytest.mark.parametrize("text,status", [
    ("8\n0 1 2 3 4 5 6 7\n", True),            # taskLoad_goodExample.txt
    ("4\n0 0 0 0\n", False),                    # taskLoadWithRepetitiveElements.txt
    ("4\n0 1 2 3 4\n", False),                  # taskLoadWithMoreThanNIndexes.txt
    ("4\n0 1\n", None),                         # taskLoadWithLessThanNIndexes.txt -> throws
    ("x\n0\n", None),
    ("0\n", None),
    ("2\n0 99\n", None),
    ("2\n0 1a\n", None),
])
def test_task_files(tmp_path, text, status):
    cfg = write(tmp_path, "c.json", json.dumps(CONFIG))
    s = load_host(write(tmp_path, "good.scn", GOOD_SCENE), cfg)
    tasks = write(tmp_path, "t.txt", text)
    if status is None:
        with pytest.raises(q.QmcrtError):
            s.load_tasks(tasks)
        with pytest.raises(ValueError):
            scene_text.parse_tasks(text, s.num_heliostats, lambda h: s.heliostat(h)["grid"])
        return
    hs, grids, st = s.load_tasks(tasks)
    assert st == status
    oh, og, ost = scene_text.parse_tasks(text, s.num_heliostats, lambda h: s.heliostat(h)["grid"])
    assert (hs, grids, st) == (oh, og, ost)


def test_task_loader_records_grid_ids(tmp_path):
    # TaskLoader.cpp:182 inserts the heliostat's grid id into the receiver set
    cfg = write(tmp_path, "c.json", json.dumps(CONFIG))
    s = load_host(write(tmp_path, "good.scn", GOOD_SCENE), cfg)
    _, grids, _ = s.load_tasks(write(tmp_path, "t.txt", "2\n0 5\n"))
    assert grids == [0, 1]


# ---- geometry: product == oracle, bit for bit ------------------------------------
def test_geometry_synthetic_small(tmp_path):
    f = synth.small_field(tmp_path, seed=3)
    assert_same_geometry(load_host(f.scene, f.config), oracle.OracleScene.from_files(f.scene, f.config))


def test_geometry_synthetic_large(tmp_path):
    f = synth.large_field(tmp_path, seed=1, num_heliostats=96, helio_pixel=0.2)
    p = load_host(f.scene, f.config)
    o = oracle.OracleScene.from_files(f.scene, f.config)
    assert_same_geometry(p, o)
    assert p.receiver(0)["width"] == 1257 and p.receiver(0)["height"] == 600


def test_set_sun_equals_loading_with_that_sun(tmp_path):
    # qmcrt_scene_set_sun re-runs the sun-dependent half of processScene: the
    # re-oriented field must equal, bit for bit, a field loaded with that sun
    # in its configuration (and therefore the oracle's).
    import json

    f = synth.large_field(tmp_path, seed=4, num_heliostats=40, helio_pixel=0.25)
    cfg = json.loads(Path(f.config).read_text())
    for sun in ([0.3, -0.8, 0.52], [-0.1, -0.95, -0.3]):
        cfg2 = dict(cfg, sun_dir=sun)
        c2 = tmp_path / f"cfg_{sun[0]}.json"
        c2.write_text(json.dumps(cfg2))
        moved = load_host(f.scene, f.config)
        moved.set_sun(sun)
        assert_same_geometry(moved, oracle.OracleScene.from_files(f.scene, c2))


def test_geometry_full_large_field_counts(tmp_path):
    f = synth.large_field(tmp_path)
    p = load_host(f.scene, f.config)
    assert p.num_heliostats == 624
    assert p.heliostat(0)["num_facets"] == 300664
    assert p.info.total_facets == 624 * 300664
    assert p.pool_size == 128 * 2048


def test_geometry_golden_cases():
    for cfg in sorted(GOLDEN.glob("cfg_*.json")):
        name = cfg.stem[4:]
        from tests.golden import make_golden as mg

        scn = mg.REF / mg.CASES[name][0]
        if not scn.exists():
            pytest.skip("reference scene files not available")
        assert_same_geometry(load_host(scn, cfg), oracle.OracleScene.from_files(scn, cfg))


def test_host_only_scene_refuses_device_calls(tmp_path):
    f = synth.small_field(tmp_path, helio_pixel=0.5)
    s = load_host(f.scene, f.config)
    with pytest.raises(q.QmcrtError) as e:
        s.trace([0])
    assert e.value.code == 4


# ---- output ------------------------------------------------------------------------
def test_save_text_format(tmp_path):
    data = np.array([[0.0, 1.234, 5e-6], [2.0, 3.14159, 0.006]], np.float32)
    mx = q.save_text(tmp_path / "img.txt", data)
    lines = (tmp_path / "img.txt").read_text().splitlines()
    # top row of the file is the last image row (ImageSaver.cpp:30-31)
    assert lines == ["2.00,3.14,0.01", "0,1.23,0"]
    assert mx == np.float32(3.14159)


def test_save_text_matches_reference(tmp_path):
    from oracle import refhost

    if not refhost.available():
        pytest.skip("reference host library not built")
    rng = np.random.default_rng(0)
    data = (rng.random((37, 23)) * 50).astype(np.float32)
    data[rng.random(data.shape) < 0.4] = 0
    data[3, 4] = 9.99e-6
    a = q.save_text(tmp_path / "a.txt", data)
    b = refhost.save_text(tmp_path / "b.txt", data)
    assert (tmp_path / "a.txt").read_text() == (tmp_path / "b.txt").read_text()
    assert a == b


# ---- the C ABI -----------------------------------------------------------------------
def test_library_exports_every_declared_symbol():
    header = "".join(p.read_text() for p in sorted((ROOT / "include").glob("*.h")))
    names = set(re.findall(r"\b(qmcrt_[a-z0-9_]+)\s*\(", header))
    assert len(names) >= 30 and "qmcrt_microbench_atomics_replay" in names
    lib = ctypes.CDLL(str(q.LIB_PATH))
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_errors_cross_the_boundary_as_codes(tmp_path):
    lib = q.load()
    h = ctypes.c_void_p()
    rc = lib.qmcrt_scene_load(b"/nonexistent.scn", b"/nonexistent.json", -1, 0, ctypes.byref(h))
    assert rc == 2 and not h.value
    assert b"doesn't exist" in lib.qmcrt_last_error()
    assert lib.qmcrt_smooth(None, 4, 4, 1, 0.1, None) == 1
    assert lib.qmcrt_last_error() != b""


def test_injected_allocation_failure_returns_a_status(tmp_path):
    """An allocation that fails (here injected at the C ABI's allocation gate)
    comes back as QMCRT_ERR_NOMEM with a message, where the reference calls
    exit(1) (Util/check_cuda.h:18-27); the library stays usable after it."""
    lib = q.load()
    f = synth.small_field(tmp_path, seed=0, helio_pixel=0.5)
    h = ctypes.c_void_p()
    try:
        assert lib.qmcrt_debug_fail_allocations(0) == 0
        rc = lib.qmcrt_scene_load(str(f.scene).encode(), str(f.config).encode(), -1, 0, ctypes.byref(h))
        assert rc == 5 and not h.value
        assert lib.qmcrt_last_error() == b"scene state: injected allocation failure"
        # injection disarmed itself: the same call now succeeds
        assert lib.qmcrt_scene_load(str(f.scene).encode(), str(f.config).encode(), -1, 0, ctypes.byref(h)) == 0
        lib.qmcrt_scene_free(h)
        # a countdown: one allocation passes, then none is made by a host-only load
        assert lib.qmcrt_debug_fail_allocations(1) == 0
        assert lib.qmcrt_scene_load(str(f.scene).encode(), str(f.config).encode(), -1, 0, ctypes.byref(h)) == 0
        lib.qmcrt_scene_free(h)
        with pytest.raises(q.QmcrtError) as err:
            q.Scene(f.scene, f.config, device=-1)
        assert err.value.code == 5 and "injected allocation failure" in str(err.value)
    finally:
        lib.qmcrt_debug_fail_allocations(-1)


def test_allocation_failure_injected_from_the_environment(tmp_path):
    import subprocess
    import sys

    f = synth.small_field(tmp_path, seed=0, helio_pixel=0.5)
    code = ("import ctypes, sys; lib = ctypes.CDLL(sys.argv[1]); h = ctypes.c_void_p(); "
            "lib.qmcrt_last_error.restype = ctypes.c_char_p; "
            "rc = lib.qmcrt_scene_load(sys.argv[2].encode(), sys.argv[3].encode(), -1, 0, ctypes.byref(h)); "
            "print(rc, lib.qmcrt_last_error().decode())")
    env = dict(os.environ, QMCRT_INJECT_ALLOC_FAILURE="0")
    r = subprocess.run([sys.executable, "-c", code, str(q.LIB_PATH), str(f.scene), str(f.config)],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "5 scene state: injected allocation failure"


def test_pipeline_executable_rejects_bad_arguments(tmp_path):
    import subprocess

    exe = q.executable()
    r = subprocess.run([str(exe), "-c", str(tmp_path / "x.txt")], capture_output=True, text=True)
    assert r.returncode != 0
    assert "suffix" in r.stderr


def test_uneven_fields_load_with_the_documented_shapes(tmp_path):
    counts, types = [], []
    for k in range(16):
        f = synth.uneven_field(tmp_path, k, seed=0, helio_pixel=1.0)
        s = q.Scene(f.scene, f.config, device=-1)
        assert 200 <= s.num_heliostats <= 2500
        side = s.heliostat(0)["size"][0]
        assert 6.0 <= side <= 12.0
        assert s.receiver(0)["type"] == k % 2
        counts.append(s.num_heliostats)
        types.append(s.receiver(0)["type"])
    assert len(set(counts)) > 8 and set(types) == {0, 1}
    # seeded: the same index and seed write the same scene
    a = synth.uneven_field(tmp_path / "a", 3, seed=0).scene.read_text()
    assert a == synth.uneven_field(tmp_path / "b", 3, seed=0).scene.read_text()


def build_facade_program(tmp_path) -> Path:
    """tests/facade_main.cpp compiled with g++ against include/qmcrt_facade.hpp, linked with libqmcrt.so."""
    import subprocess

    exe = tmp_path / "facade_main"
    lib_dir = q.LIB_PATH.parent
    r = subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "facade_main.cpp"),
                        f"-L{lib_dir}", "-lqmcrt", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def run_facade(exe, files, out_dir, device: int) -> dict:
    import subprocess

    r = subprocess.run([str(exe), str(files.scene), str(files.config), str(files.tasks), str(out_dir), str(device)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return dict(kv.split("=") for kv in r.stdout.split())


def test_cpp_facade_with_the_reference_names_host_only(tmp_path):
    files = synth.small_field(tmp_path, seed=1, helio_pixel=0.5)
    res = run_facade(build_facade_program(tmp_path), files, tmp_path, -1)
    assert res["fields"] == "10" and res["heliostats"] == "50"
    assert res["tasks_ok"] == "1" and res["tasks"] == "50" and res["receivers"] == "1"
