"""Generate tests/golden/work_per_ray_624field.json: the reference algorithm's
work per ray on the benchmark field, counted by the CPU oracle.

The oracle restates the reference's per-ray routine
(QuasiMonteCarloRayTracing/RectangleReceiverRectangleGridRayTracing.cu:6-41,
CylinderReceiverRectangleGridRayTracing.cu:6-40, Grid/rectGridDDA.cu:7-119,
Util/global_function.cuh:101-136) and counts, on a fixed subsample (every
4001st micro-facet x 8 light indexes of the seed-0 624-heliostat field, with
the sun-shape and slope-error pools and facet offsets the tracer generates
for seed 0), the parallelogram tests reaching each stage, the grid cells
visited and the receiver hits.  The algorithmic FP32 flops per ray credit
23 / 6 / 15 / 6 flops per stage of rayParallelogramIntersect, 20 per cell
step, 70 for sampling, perturbation and reflection and 55 for the cylinder
test when reached.  bench.py reads the frozen figures for its roofline.

It also measures how the flux deposits of one warp fall (`deposits`): on
every 13th heliostat x a 2,048-facet range x light indexes 0-31, grouped as
the tracer's warps take them (an iteration = the 32 light indexes of one
facet, a chunk = 64 iterations), the receiver hits per iteration and per
chunk and how many distinct pixels they land in.  Merging a warp's deposits
into one atomic per distinct pixel (or a per-warp tile) can only save the
difference.

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


def deposits(o, dirs, pert, seed: int, stride: int = 13, facets: int = 2048, chunk_iters: int = 64) -> dict:
    """Receiver hits and distinct pixels per warp iteration and warp chunk."""
    from oracle.cpu_baseline import scene_offsets

    it_hits, it_px, ch_hits, ch_px = [], [], [], []
    for h in range(0, o.num_heliostats, stride):
        nf = o.heliostat(h)["num_facets"]
        fb = nf // 2 - facets // 2
        offs = scene_offsets(o, seed, [h])
        rec = o.trace([h], dirs, pert, offs, 0, 32, record=(h, fb, fb + facets), images=False)["records"]
        rec = rec.reshape(facets, 32)
        for row in rec:
            hit = row[row >= 0]
            it_hits.append(hit.size)
            it_px.append(np.unique(hit).size)
        for c in range(0, facets, chunk_iters):
            hit = rec[c:c + chunk_iters].ravel()
            hit = hit[hit >= 0]
            ch_hits.append(hit.size)
            ch_px.append(np.unique(hit).size)
    return {"per_iteration": {"hits": float(np.mean(it_hits)), "distinct_pixels": float(np.mean(it_px))},
            "per_chunk": {"hits": float(np.mean(ch_hits)), "distinct_pixels": float(np.mean(ch_px))},
            "sample": f"every {stride}th heliostat x {facets} facets x light indexes 0-31"}


def census(files, lights: int = 8, stride: int = 4001, seed: int = 0) -> dict:
    from oracle.cpu_baseline import scene_offsets, scene_pools

    o = orc.OracleScene.from_files(files.scene, files.config)
    dirs, pert = scene_pools(o, seed)
    offs = scene_offsets(o, seed, range(o.num_heliostats))
    res = o.trace(list(range(o.num_heliostats)), dirs, pert, offs, 0, lights, facet_stride=stride, images=False)
    c = res["counters"]
    n = max(c["rays"], 1)
    per = {k: c[k] / n for k in ("tests_det", "tests_u", "tests_v", "tests_t", "cells", "hit", "shadowed", "blocked",
                                 "missed")}
    reach_receiver = (c["hit"] + c["missed"]) / n
    per["flops"] = (23 * per["tests_det"] + 6 * per["tests_u"] + 15 * per["tests_v"] + 6 * per["tests_t"]
                    + 20 * per["cells"] + 70 + 55 * reach_receiver)
    per["rays_sampled"] = n
    per["deposits"] = deposits(o, dirs, pert, seed)
    return per


def main() -> None:
    files = synth.large_field(Path(tempfile.mkdtemp(prefix="census_")), seed=0)
    per = census(files)
    per["field"] = "synth.large_field(seed=0): 624 focus-flat heliostats, cylinder receiver"
    per["sample"] = ("every 4001st micro-facet x light indexes 0-7; the tracer's seed-0 Buie CSR 0.1 and 2.9 mrad "
                     "slope-error pools and facet offsets")
    OUT.write_text(json.dumps(per, indent=1) + "\n")
    print(OUT, per["flops"])


if __name__ == "__main__":
    main()
