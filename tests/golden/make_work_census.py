"""Generate tests/golden/work_per_ray_624field.json: the reference algorithm's
work per ray on the benchmark field, counted by the CPU oracle.

The oracle restates the reference's per-ray routine
(QuasiMonteCarloRayTracing/RectangleReceiverRectangleGridRayTracing.cu:6-41,
CylinderReceiverRectangleGridRayTracing.cu:6-40, Grid/rectGridDDA.cu:7-119,
Util/global_function.cuh:101-136) and counts, on a fixed subsample (every
4001st micro-facet x 8 light indexes of the seed-0 624-heliostat field with
seeded pools), the parallelogram tests reaching each stage, the grid cells
visited and the receiver hits.  The algorithmic FP32 flops per ray credit
23 / 6 / 15 / 6 flops per stage of rayParallelogramIntersect, 20 per cell
step, 70 for sampling, perturbation and reflection and 55 for the cylinder
test when reached.  bench.py reads the frozen figures for its roofline.

Usage:  python tests/golden/make_work_census.py
"""
from __future__ import annotations

import json
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as orc  # noqa: E402
from solarenergy_chier_b200 import synth  # noqa: E402

OUT = Path(__file__).resolve().parent / "work_per_ray_624field.json"


def census(files, lights: int = 8, stride: int = 4001) -> dict:
    o = orc.OracleScene.from_files(files.scene, files.config)
    P = o.pool_size
    rng = np.random.default_rng(5)
    th = 0.00465 * np.sqrt(rng.random(P))
    ph = 2 * np.pi * rng.random(P)
    dirs = np.stack([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)], 1).astype(np.float32)
    pert = np.tile(np.array([0, 1, 0], np.float32), (P, 1))
    offs = {h: rng.integers(0, P, o.heliostat(h)["num_facets"] + 1).astype(np.int32) for h in range(o.num_heliostats)}
    res = o.trace(list(range(o.num_heliostats)), dirs, pert, offs, 0, lights, facet_stride=stride, images=False)
    c = res["counters"]
    n = max(c["rays"], 1)
    per = {k: c[k] / n for k in ("tests_det", "tests_u", "tests_v", "tests_t", "cells", "hit", "shadowed", "blocked",
                                 "missed")}
    reach_receiver = (c["hit"] + c["missed"]) / n
    per["flops"] = (23 * per["tests_det"] + 6 * per["tests_u"] + 15 * per["tests_v"] + 6 * per["tests_t"]
                    + 20 * per["cells"] + 70 + 55 * reach_receiver)
    per["rays_sampled"] = n
    return per


def main() -> None:
    files = synth.large_field(Path(tempfile.mkdtemp(prefix="census_")), seed=0)
    per = census(files)
    per["field"] = "synth.large_field(seed=0): 624 focus-flat heliostats, cylinder receiver"
    per["sample"] = "every 4001st micro-facet x light indexes 0-7, seeded pools"
    OUT.write_text(json.dumps(per, indent=1) + "\n")
    print(OUT, per["flops"])


if __name__ == "__main__":
    main()
