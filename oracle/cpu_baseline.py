"""CPU ORACLE - test infrastructure only: the CPU baseline of bench.py and the
checker of its accuracy figures.

Times the reference's own per-ray routine (oracle/_ref/libref_host.so: its
host code compiled from the reference tree, OpenMP over every host core) -
or, when that library is absent, the oracle's restatement - on a bounded
sample of a scene: every `stride`-th micro-facet of every heliostat for a
number of light indexes chosen so the run lasts about `seconds`.  The rays
are the GPU arm's workload: the sun-shape and slope-error pools the tracer
generates at load with the same seed (restated here from the generator's
definition: Buie from scrambled-Sobol uniforms through the reference's
inverse CDF, Box-Muller slope errors; within 2e-7 of the device's) and the
same seeded facet offsets.

With an accuracy input (npz written by bench.py: the tracer's own pools, its
flux image, FP64 total power and per-ray outcome codes on a sample of the
same field), it also checks those against the CPU oracle in float (the
reference's host arithmetic, which its own code pins bit for bit) and in
FP64, untimed, and reports the errors.

Runs in its own process so that no CUDA library of the caller shares its
symbol namespace:

    python -m oracle.cpu_baseline scene config seconds [seed] [accuracy.npz]

Prints one JSON object.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np


def scene_pools(o, seed: int):
    """The sun-shape (Buie, the configuration's CSR) and slope-error pools the
    tracer generates for `seed` at scene load (qmcrt_scene_load: pool
    generator seeds mix32(seed * 2654435761 + 1) and + 2), restated with the
    oracle's Sobol and Buie routines."""
    from oracle import oracle as orc

    P = o.pool_size
    cfg = o.config
    mix = orc.mix32
    seed_sun = mix((seed * 2654435761 + 1) & 0xFFFFFFFF)
    seed_slope = mix((seed * 2654435761 + 2) & 0xFFFFFFFF)
    xy = orc.sobol2(seed_sun, 0, P)
    uf = ((xy[:, 0] >> 8).astype(np.float32) * np.float32(1.0 / 16777216.0)).astype(np.float32)
    theta = orc.buie_theta(cfg["csr"], cfg["inverse_transform_sampling_groups"], uf).astype(np.float32)
    phi = ((xy[:, 1] >> 8).astype(np.float32) * np.float32(1.0 / 16777216.0) * np.float32(2 * 3.141592654))
    dirs = np.stack([np.sin(theta) * np.cos(phi), np.cos(theta), np.sin(theta) * np.sin(phi)], 1).astype(np.float32)
    xy = orc.sobol2(seed_slope, 0, P).astype(np.float64)
    u, v = (xy[:, 0] + 0.5) / 2 ** 32, (xy[:, 1] + 0.5) / 2 ** 32
    r = np.sqrt(-2 * np.log(u))
    sigma = np.float64(np.float32(cfg["helio_disturb_std"]))
    w = np.stack([(sigma * r * np.cos(2 * np.pi * v)).astype(np.float32), np.ones(P, np.float32),
                  (sigma * r * np.sin(2 * np.pi * v)).astype(np.float32)], 1).astype(np.float64)
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    return dirs, w.astype(np.float32)


def scene_offsets(o, seed: int, heliostats):
    """The tracer's seeded facet offsets (num_facets + 1 per heliostat)."""
    from oracle import oracle as orc

    P = o.pool_size
    return {h: orc.facet_offsets(seed, h, o.heliostat(h)["num_facets"] + 1, P) for h in heliostats}


def l1(a, b):
    return float(np.abs(a - b).sum() / b.sum())


def accuracy(scene_path: str, config_path: str, path: str) -> dict:
    """Errors of the tracer's outputs on a sample of the field, against the
    CPU oracle in float (the reference's host arithmetic) and in FP64."""
    from oracle import oracle as orc

    d = np.load(path)
    dirs, pert = d["dirs"], d["pert"]
    seed = int(d["seed"])
    f32 = orc.OracleScene.from_files(scene_path, config_path)
    f64 = orc.OracleScene.from_files(scene_path, config_path, precision=64)
    out = {}
    ids = [int(h) for h in d["flux_ids"]]
    lights = int(d["flux_lights"])
    offs = scene_offsets(f32, seed, ids)
    t0 = time.time()
    a32 = f32.trace(ids, dirs, pert, offs, 0, lights)
    a64 = f64.trace(ids, dirs, pert, offs, 0, lights)
    img = d["flux_image"].astype(np.float64)
    total = float(d["flux_power"])
    r32, r64 = a32["images"][0], a64["images"][0]
    t32, t64 = float(a32["power"].sum()), float(a64["power"].sum())
    out["flux"] = {
        "sample": f"heliostats {ids[0]}..{ids[-1]} step {ids[1] - ids[0] if len(ids) > 1 else 1} ({len(ids)}) x every "
                  f"facet x light indexes 0-{lights - 1}: {a32['counters']['rays']} rays",
        "flux_l1_vs_fp64": l1(img, r64), "reference_arithmetic_flux_l1_vs_fp64": l1(r32, r64),
        "flux_l1_vs_reference_arithmetic": l1(img, r32),
        "power_rel_vs_fp64": abs(total - t64) / t64, "reference_arithmetic_power_rel_vs_fp64": abs(t32 - t64) / t64,
        "power_rel_vs_reference_arithmetic": abs(total - t32) / t32}
    rec_ids, rec_fb = d["rec_ids"], d["rec_facet_begin"]
    nfac, rl = int(d["rec_facets"]), int(d["rec_lights"])
    codes = d["rec_codes"].reshape(len(rec_ids), -1)
    n = same = dec = dec64 = ref_dec64 = 0
    for k, h in enumerate(rec_ids):
        h, fb = int(h), int(rec_fb[k])
        o1 = scene_offsets(f32, seed, [h])
        rec = (h, fb, fb + nfac)
        want = f32.trace([h], dirs, pert, o1, 0, rl, record=rec, images=False, record_only=True)["records"]
        w64 = f64.trace([h], dirs, pert, o1, 0, rl, record=rec, images=False, record_only=True)["records"]
        got = codes[k]
        n += got.size
        same += int(np.count_nonzero(got == want))
        dec += int(np.count_nonzero((got >= 0) == (want >= 0)))
        dec64 += int(np.count_nonzero((got >= 0) == (w64 >= 0)))
        ref_dec64 += int(np.count_nonzero((want >= 0) == (w64 >= 0)))
    out["per_ray"] = {
        "sample": f"{len(rec_ids)} heliostats x {nfac} facets x light indexes 0-{rl - 1}: {n} rays",
        "hit_decision_agreement_vs_reference_arithmetic": dec / n,
        "outcome_agreement_vs_reference_arithmetic": same / n,
        "hit_decision_agreement_vs_fp64": dec64 / n,
        "reference_arithmetic_hit_decision_agreement_vs_fp64": ref_dec64 / n}
    out["check_seconds"] = round(time.time() - t0, 1)
    return out


def run(scene_path: str, config_path: str, seconds: float, seed: int = 0) -> dict:
    from oracle import oracle as orc
    from oracle import refhost

    kind = "reference" if refhost.available() else "port"
    threads = len(os.sched_getaffinity(0))
    if kind == "reference":
        r = refhost.RefScene(scene_path, config_path)
    else:
        r = orc.OracleScene.from_files(scene_path, config_path)
    o = orc.OracleScene.from_files(scene_path, config_path)
    nh = o.num_heliostats
    nf = [o.heliostat(h)["num_facets"] for h in range(nh)]
    L = o.config["num_per_sunshape_group"]
    dirs, pert = scene_pools(o, seed)
    offs = scene_offsets(o, seed, range(nh))
    ids = list(range(nh))
    stride = max(1, sum(nf) // 20000)

    def go(lights):
        t0 = time.time()
        if kind == "reference":
            res = r.trace(ids, dirs, pert, offs, L, 0, lights, facet_stride=stride, images=False)
        else:
            res = r.trace(ids, dirs, pert, offs, 0, lights, facet_stride=stride, images=False)
        return res["counters"]["rays"], time.time() - t0

    _, dt1 = go(1)
    _, dt4 = go(4)
    per_light = max((dt4 - dt1) / 3.0, 1e-4)
    lights = int(max(1, min(L, seconds / per_light)))
    rays, dt = go(lights)
    return {"value": rays / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": kind,
            "sample": f"every {stride}th micro-facet of all {nh} heliostats x {lights} light index(es): "
                      f"{rays} rays in {dt:.1f} s; the GPU arm's Buie CSR {o.config['csr']:g} sun-shape pool, "
                      f"{o.config['helio_disturb_std'] * 1e3:g} mrad slope-error pool and facet offsets (seed {seed})"}


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    seed = int(sys.argv[4]) if len(sys.argv) > 4 else 0
    res = run(sys.argv[1], sys.argv[2], float(sys.argv[3]), seed)
    if len(sys.argv) > 5:
        res["accuracy"] = accuracy(sys.argv[1], sys.argv[2], sys.argv[5])
    print(json.dumps(res))
