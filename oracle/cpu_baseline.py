"""CPU ORACLE - test infrastructure only: the CPU baseline of bench.py.

Times the reference's own per-ray routine (oracle/_ref/libref_host.so: its
host code compiled from the reference tree, OpenMP over every host core) -
or, when that library is absent, the oracle's restatement - on a bounded
sample of a scene: every `stride`-th micro-facet of every heliostat for a
number of light indexes chosen so the run lasts about `seconds`.

Runs in its own process (python -m oracle.cpu_baseline scene config seconds)
so that no CUDA library of the caller shares its symbol namespace.
Prints one JSON object.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np


def run(scene_path: str, config_path: str, seconds: float) -> dict:
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
    P = o.pool_size
    L = o.config["num_per_sunshape_group"]
    rng = np.random.default_rng(9)
    th = 0.00465 * np.sqrt(rng.random(P))
    ph = 2 * np.pi * rng.random(P)
    dirs = np.stack([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)], 1).astype(np.float32)
    pert = np.tile(np.array([0, 1, 0], np.float32), (P, 1))
    offs = {h: rng.integers(0, P, nf[h] + 1).astype(np.int32) for h in range(nh)}
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
                      f"{rays} rays in {dt:.1f} s"}


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    print(json.dumps(run(sys.argv[1], sys.argv[2], float(sys.argv[3]))))
