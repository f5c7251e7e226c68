"""Generate tests/golden/*.npz from the reference's own code.

Runs oracle/_ref/libref_host.so (the reference tree's host code built by
oracle/build_ref.py) on the reference's example and test scenes and on a
small synthetic field, with seeded sample pools and facet offsets, and
stores its outputs as golden vectors:

  geometry_<case>.npz   receivers, heliostat normals, grid cell lists,
                        sub-heliostat tables, micro-facets
  trace_<case>.npz      pools, offsets, per-ray outcome codes, images
                        (sparse), per-heliostat power for 64 light indexes,
                        traced with cfg_<case>.json (the case's configuration
                        with two sun-shape groups, to keep the pools small)
  smooth.npz            trimmed-mean outputs on seeded images
  buie.npz              Buie tables and inverse-CDF samples

Usage (needs the reference tree, i.e. this container):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import build_ref, refhost  # noqa: E402
from tests.golden.fixtures import offsets_for  # noqa: E402
from solarenergy_chier_b200 import synth  # noqa: E402

OUT = Path(__file__).resolve().parent
REF = build_ref.REF

CASES = {
    "qmcrt_rect": ("Tests/QuasiMonteCarloRayTracingTests/test_file/test_scene.scn",
                   "Tests/QuasiMonteCarloRayTracingTests/test_file/test_configuration.json"),
    "qmcrt_cyl": ("Tests/QuasiMonteCarloRayTracingTests/test_file/test_scene_cylinder_receiver.scn",
                  "Tests/QuasiMonteCarloRayTracingTests/test_file/test_configuration2.json"),
    "focusflat_test": ("Tests/DataStructureTests/test_file/test_scene_good_for_focusFlatRectangleHelio.scn",
                       "Tests/DataStructureTests/test_file/test_configuration.json"),
    "ps10_4x7": ("InputFiles/PS10_typical/PS10_typical_4x7_scene.scn",
                 "InputFiles/PS10_typical/PS10_typical_4x7_configuration.json"),
    "two_receivers": ("InputFiles/CompleteInputFilesExample/twoReceiverScene.scn",
                      "InputFiles/CompleteInputFilesExample/twoReceiverConfiguration.json"),
    "focusflat_example": ("InputFiles/FocusFlatRectangleHeliostatInputs/focusflat_example_scene.scn",
                          "InputFiles/FocusFlatRectangleHeliostatInputs/focusflat_example_configuration.json"),
}


def seeded_pools(pool_size: int, seed: int, half_angle: float = 0.00465, sigma: float = 0.002):
    """Sun-shape and slope-error pools drawn with numpy (seeded): directions
    uniform over a disc of `half_angle`, slope normals normalize(N(0,s),1,N(0,s))."""
    rng = np.random.default_rng(seed)
    th = half_angle * np.sqrt(rng.random(pool_size))
    ph = 2 * np.pi * rng.random(pool_size)
    dirs = np.stack([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)], 1).astype(np.float32)
    x = (rng.standard_normal(pool_size) * sigma).astype(np.float32)
    z = (rng.standard_normal(pool_size) * sigma).astype(np.float32)
    p = np.stack([x, np.ones(pool_size, np.float32), z], 1).astype(np.float64)
    pert = (p / np.linalg.norm(p, axis=1, keepdims=True)).astype(np.float32)
    return dirs, pert


def geometry(name: str, r: refhost.RefScene) -> None:
    out = {"counts": np.array([r.num_receivers, r.num_grids, r.num_heliostats], np.int32)}
    for i in range(r.num_receivers):
        rc = r.receiver(i)
        out[f"recv{i}_size"] = np.array([rc["type"], rc["width"], rc["height"]], np.int32)
        out[f"recv{i}_vertices"] = rc["vertices"]
        out[f"recv{i}_pixel_length"] = np.float32(rc["pixel_length"])
    for g in range(r.num_grids):
        gd = r.grid(g)
        out[f"grid{g}_cells"] = np.array(gd["cells"], np.int32)
        out[f"grid{g}_index"] = gd["index"]
        out[f"grid{g}_match"] = gd["match"]
        out[f"grid{g}_vertices"] = gd["vertices"]
    hs = [r.heliostat(h) for h in range(r.num_heliostats)]
    out["helio_ints"] = np.array([[h["type"], h["grid"], h["num_facets"], h["num_sub"], h["sub_begin"]] for h in hs],
                                 np.int32)
    out["helio_normals"] = np.array([h["normal"] for h in hs], np.float32)
    for h in range(min(r.num_heliostats, 3)):
        o, n = r.facets(h)
        step = max(1, len(o) // 4096)
        out[f"facets{h}_index"] = np.arange(0, len(o), step, dtype=np.int32)
        out[f"facets{h}_origins"] = o[::step]
        out[f"facets{h}_normals"] = n[::step]
    np.savez_compressed(OUT / f"geometry_{name}.npz", **out)


def small_pool_config(config_path: Path, name: str) -> Path:
    """The case's configuration with num_of_sunshape_groups = 2, written next
    to the fixtures, so that the pools stored with the golden outputs stay small."""
    import json
    cfg = json.loads(Path(config_path).read_text())
    cfg["num_of_sunshape_groups"] = 2
    out = OUT / f"cfg_{name}.json"
    out.write_text(json.dumps(cfg, indent=2) + "\n")
    return out


def trace(name: str, r: refhost.RefScene, scene_path: Path, config_path: Path, lights: int, facets: int) -> None:
    import json
    cfg = json.loads(Path(config_path).read_text())
    groups = cfg.get("num_of_sunshape_groups", 128)
    per_group = cfg.get("num_per_sunshape_group", 2048)
    P = groups * per_group
    dirs, pert = seeded_pools(P, 7)
    nf = [r.heliostat(h)["num_facets"] for h in range(r.num_heliostats)]
    offs = offsets_for(nf, P, 11)
    out = {"pool_dirs": dirs, "pool_pert": pert, "lights": np.int32(lights), "offset_seed": np.int64(11)}
    ids = list(range(min(r.num_heliostats, 4)))
    out["ids"] = np.array(ids, np.int32)
    for h in ids:
        fe = min(nf[h], facets)
        res = r.trace([h], dirs, pert, offs, per_group, 0, lights, record=(h, 0, fe))
        out[f"records{h}"] = res["records"]
        out[f"power{h}"] = np.float64(res["power"][h])
        for k, img in enumerate(res["images"]):
            flat = img.ravel()
            nz = np.nonzero(flat)[0].astype(np.int32)
            out[f"image{h}_{k}_index"] = nz
            out[f"image{h}_{k}_value"] = flat[nz]
        out[f"counters{h}"] = np.array([res["counters"][k] for k in ("rays", "shadowed", "blocked", "missed", "hit",
                                                                    "clamped")], np.int64)
    np.savez_compressed(OUT / f"trace_{name}.npz", **out)


def main() -> None:
    if not build_ref.available():
        raise SystemExit("reference tree not found; golden vectors can only be regenerated where it is mounted")
    build_ref.build()
    for name, (scn, cfg) in CASES.items():
        r = refhost.RefScene(REF / scn, REF / cfg)
        geometry(name, r)
        small = small_pool_config(REF / cfg, name)
        r = refhost.RefScene(REF / scn, small)
        trace(name, r, REF / scn, small, lights=64, facets=256)
        print("wrote", name)
    tmp = OUT / "_tmp_small"
    f = synth.small_field(tmp, seed=0, helio_pixel=0.25, groups=16, per_group=256)
    r = refhost.RefScene(f.scene, f.config)
    geometry("synth_small", r)
    trace("synth_small", r, f.scene, f.config, lights=32, facets=256)
    for p in sorted(tmp.iterdir()):
        (OUT / ("synth_small_" + p.name.split("_", 1)[1])).write_text(p.read_text())
        p.unlink()
    tmp.rmdir()
    print("wrote synth_small")
    rng = np.random.default_rng(3)
    sm = {}
    for k, (h, w, rad, ratio) in enumerate([(40, 57, 1, 0.17), (33, 48, 5, 0.05), (20, 20, 2, 0.2), (9, 13, 3, 0.1)]):
        img = (rng.random((h, w)) * 100).astype(np.float32)
        img[rng.random((h, w)) < 0.3] = 0.0
        img[5, :] = 7.0  # ties
        sm[f"in{k}"] = img
        sm[f"out{k}"] = refhost.smooth(img, rad, ratio)
        sm[f"params{k}"] = np.array([rad, ratio], np.float64)
    np.savez_compressed(OUT / "smooth.npz", **sm)
    bu = {}
    for k, (csr, groups) in enumerate([(0.1, 1024), (0.05, 64), (0.3, 512)]):
        t = refhost.buie_table(csr, groups)
        for key, v in t.items():
            bu[f"{key}{k}"] = np.asarray(v)
        u = np.concatenate([np.linspace(0, 1, 4001, dtype=np.float32), rng.random(4000).astype(np.float32)])
        bu[f"u{k}"] = u
        bu[f"theta{k}"] = refhost.buie_theta(csr, groups, u)
        bu[f"params{k}"] = np.array([csr, groups], np.float64)
    np.savez_compressed(OUT / "buie.npz", **bu)
    print("wrote smooth, buie")


if __name__ == "__main__":
    main()
