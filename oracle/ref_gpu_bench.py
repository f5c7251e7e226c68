"""REFERENCE TIMING HARNESS - benchmark infrastructure only.

Times the reference's own CUDA tracer (oracle/_ref/libref_gpu.so, built from
the reference tree by build_ref.py) on the same GPU, in its own process:

  pipeline   QuasiMonteCarloRayTracer::rayTracing per heliostat, unchanged
             (per-heliostat vertex-table rebuild, micro-facet kernels,
             cuRAND offsets, allocations and synchronisations included);
  kernel     the Rectangle/CylinderReceiverRectangleGridRayTracing launch
             alone, arguments prepared outside the timed region.

    python -m oracle.ref_gpu_bench scene.scn config.json ids...   -> one JSON line

The reference reads the facet offset of facet f+1 for the last facet; with
fewer facets than pool samples that read is one element past its buffer, so
this harness refuses heliostats with fewer micro-facets than the pool holds.
"""
from __future__ import annotations

import ctypes
import json
import sys
from pathlib import Path

LIB = Path(__file__).resolve().parent / "_ref" / "libref_gpu.so"


def main(argv):
    scene, config, ids = argv[0], argv[1], [int(x) for x in argv[2:]]
    if not LIB.exists():
        print(json.dumps({"unavailable": "oracle/_ref/libref_gpu.so was not built"}))
        return 0
    L = ctypes.CDLL(str(LIB))
    L.refgpu_last_error.restype = ctypes.c_char_p
    counts = (ctypes.c_int * 3)()
    rc = L.refgpu_load(scene.encode(), config.encode(), counts)
    if rc != 0:
        print(json.dumps({"unavailable": "reference load failed: " + L.refgpu_last_error().decode()}))
        return 0
    lights = L.refgpu_lights_per_group()
    pool = L.refgpu_pool_size()
    facets = []
    for h in ids:
        n = L.refgpu_num_facets(h)
        if n < pool:
            print(json.dumps({"unavailable": f"heliostat {h} has {n} facets < pool {pool}: the reference "
                                             "would read past its offset buffer"}))
            return 0
        facets.append(n)
    arr = (ctypes.c_int * len(ids))(*ids)
    ms_k = ctypes.c_float()
    rc = L.refgpu_trace_kernels(arr, len(ids), ctypes.byref(ms_k))
    if rc != 0:
        print(json.dumps({"unavailable": "kernel timing failed: " + L.refgpu_last_error().decode()}))
        return 0
    ms_p = ctypes.c_float()
    rc = L.refgpu_trace_pipeline(arr, len(ids), ctypes.byref(ms_p))
    if rc != 0:
        print(json.dumps({"unavailable": "pipeline timing failed: " + L.refgpu_last_error().decode()}))
        return 0
    rays = sum(facets) * lights
    print(json.dumps({"heliostats": ids, "rays": rays, "kernel_ms": ms_k.value, "pipeline_ms": ms_p.value,
                      "kernel_mrays_s": rays / (ms_k.value / 1e3) / 1e6,
                      "pipeline_mrays_s": rays / (ms_p.value / 1e3) / 1e6}))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
