"""REFERENCE PARITY HARNESS - test infrastructure only.

Runs the reference's own CUDA tracer (oracle/_ref/libref_gpu.so, built from
the reference tree by build_ref.py) with injected sample pools and facet
offsets, in its own process (the reference keeps one scene per process in
singletons), and saves its receiver images:

    python -m oracle.ref_gpu_parity scene.scn config.json inputs.npz out.npz [per-heliostat | record]

inputs.npz: dirs (P, 3), pert (P, 3) float32 and, per traced heliostat h,
offsets_<h> (num_facets + 1 int32).  out.npz: image<r> per receiver (all
listed heliostats accumulated); with "per-heliostat", also image<r>_h<h>,
each heliostat traced alone into a cleared image; with "record", also, per
heliostat, every ray's outcome as the reference's kernel steps compute it
(refgpu_record_with_offsets: code<h> int32 - pixel index, -1 shadowed,
-2 blocked, -3 missed -, u<h>, v<h>, energy<h> float32, row-major by facet).
"""
from __future__ import annotations

import ctypes
import sys
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libref_gpu.so"


def main(argv) -> int:
    scene, config, inputs, out = argv[:4]
    L = ctypes.CDLL(str(LIB))
    L.refgpu_last_error.restype = ctypes.c_char_p
    counts = (ctypes.c_int * 3)()

    def ok(rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: {L.refgpu_last_error().decode()} ({rc})")

    ok(L.refgpu_load(scene.encode(), config.encode(), counts), "load")
    d = np.load(inputs)
    dirs = np.ascontiguousarray(d["dirs"], np.float32)
    pert = np.ascontiguousarray(d["pert"], np.float32)
    ok(L.refgpu_set_pools(dirs.ctypes.data_as(ctypes.c_void_p), pert.ctypes.data_as(ctypes.c_void_p),
                          dirs.shape[0]), "pools")
    per = len(argv) > 4 and argv[4] == "per-heliostat"
    record = len(argv) > 4 and argv[4] == "record"
    L.refgpu_num_facets.restype = ctypes.c_int
    lights = L.refgpu_lights_per_group()

    def read(r):
        w, h = ctypes.c_int(), ctypes.c_int()
        L.refgpu_image(r, None, ctypes.byref(w), ctypes.byref(h))
        img = np.zeros((h.value, w.value), np.float32)
        L.refgpu_image(r, img.ctypes.data_as(ctypes.c_void_p), ctypes.byref(w), ctypes.byref(h))
        return img

    images = {}
    keys = sorted((k for k in d.files if k.startswith("offsets_")), key=lambda k: int(k.split("_")[1]))
    total = [None] * counts[0]
    for r in range(counts[0]):
        ok(L.refgpu_clear_image(r), "clear")
    for key in keys:
        h = int(key.split("_")[1])
        o = np.ascontiguousarray(d[key], np.int32)
        ok(L.refgpu_trace_with_offsets(h, o.ctypes.data_as(ctypes.c_void_p), o.size), f"trace {h}")
        if record:
            n = (o.size - 1) * lights
            rec = {"code": np.empty(n, np.int32), "u": np.empty(n, np.float32), "v": np.empty(n, np.float32),
                   "energy": np.empty(n, np.float32)}
            ok(L.refgpu_record_with_offsets(h, o.ctypes.data_as(ctypes.c_void_p), o.size, 0, o.size - 1,
                                            *(rec[k].ctypes.data_as(ctypes.c_void_p)
                                              for k in ("code", "u", "v", "energy"))), f"record {h}")
            for k, a in rec.items():
                images[f"{k}{h}"] = a
        if per:
            for r in range(counts[0]):
                img = read(r)
                images[f"image{r}_h{h}"] = img
                total[r] = img.astype(np.float64) if total[r] is None else total[r] + img
                ok(L.refgpu_clear_image(r), "clear")
    for r in range(counts[0]):
        images[f"image{r}"] = total[r].astype(np.float32) if per else read(r)
    np.savez(out, **images)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
