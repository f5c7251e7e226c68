"""REFERENCE PIPELINE HARNESS - test infrastructure only.

The steps of RayTracingPipeline::rayTracing after scene processing
(RayTracingPipeline/RayTracingPipeline.cpp:54-102) and saveReceiverResult
(:117-142), run on the reference's own host code (oracle/_ref/libref_host.so,
built from its tree by build_ref.py): the task list read by its TaskLoader,
every listed heliostat traced by its per-ray routine with injected sample
pools and facet offsets (its pools come from a time-seeded cuRAND, which
nothing can reproduce), then, for each receiver index the task list records,
the flux map written by its ImageSaver::saveText, smoothed by its
trimmed-mean heaps (radius 5, ratio 0.05) and written again.  The images are
accumulated in float, as its atomicAdd accumulates them.  Its own process
(the reference keeps one scene per process in singletons):

    python -m oracle.ref_pipeline config.json scene.scn tasks.txt inputs.npz out_dir/

inputs.npz: dirs, pert (P x 3 float32) and offsets_<h> (num_facets + 1 int32)
for every listed heliostat.
"""
from __future__ import annotations

import os
import sys

import numpy as np


def main(argv) -> int:
    config, scene, tasks, inputs, out = argv[:5]
    from oracle import refhost

    r = refhost.RefScene(scene, config)
    ids, receivers, _ = r.load_tasks(tasks)
    d = np.load(inputs)
    offsets = {h: d[f"offsets_{h}"] for h in ids}
    L = int(d["per_group"])
    res = r.trace(ids, d["dirs"], d["pert"], offsets, L, 0, L)
    for k in receivers:
        img = res["images"][k].astype(np.float32)
        base = os.path.join(out, str(k))
        refhost.save_text(base + "_receiver_before_smooth.txt", img)
        refhost.save_text(base + "_receiver_after_smooth.txt", refhost.smooth(img, 5, 0.05))
    return 0


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    sys.exit(main(sys.argv[1:]))
