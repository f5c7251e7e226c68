"""Python side of the C ABI, mirroring the reference's entry points.

`Scene` wraps a loaded and processed scene (SolarScene + SceneConfiguration +
SceneProcessor).  The reference-named helpers below (QuasiMonteCarloRayTracer,
ImageSmoother, ImageSaver, TaskLoader, RayTracingPipeline) keep the method
names of SolarEnergy_Chier so that test and driver code reads the same.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from ._lib import SceneInfo, check, load

_pf = ctypes.POINTER(ctypes.c_float)
_pi = ctypes.POINTER(ctypes.c_int)
_pd = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _stream_handle(stream) -> ctypes.c_void_p | None:
    """Accepts None, an int handle, or an object with .cuda_stream (torch)."""
    if stream is None:
        return None
    handle = getattr(stream, "cuda_stream", stream)
    return ctypes.c_void_p(int(handle))


SUNSHAPE_BUIE = 0
SUNSHAPE_PILLBOX = 1


class Scene:
    """A loaded scene on one CUDA device (qmcrt_scene_load)."""

    def __init__(self, scene_path, config_path, device: int = 0, seed: int = 0):
        lib = load()
        handle = ctypes.c_void_p()
        check(lib.qmcrt_scene_load(str(scene_path).encode(), str(config_path).encode(), int(device),
                                   int(seed) & 0xFFFFFFFF, ctypes.byref(handle)))
        self._h = handle
        self._lib = lib
        self.device = device
        info = SceneInfo()
        check(lib.qmcrt_scene_get_info(self._h, ctypes.byref(info)))
        self.info = info

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.qmcrt_scene_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    # -- scene state --------------------------------------------------------
    @property
    def num_heliostats(self) -> int:
        return self.info.num_heliostats

    @property
    def num_receivers(self) -> int:
        return self.info.num_receivers

    @property
    def num_grids(self) -> int:
        return self.info.num_grids

    @property
    def pool_size(self) -> int:
        return self.info.pool_size

    @property
    def lights_per_group(self) -> int:
        return self.info.num_per_sunshape_group

    def receiver(self, i: int) -> dict:
        t, w, h = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        px = ctypes.c_float()
        verts = np.zeros(12, np.float32)
        normal = np.zeros(3, np.float32)
        focus = np.zeros(3, np.float32)
        check(self._lib.qmcrt_receiver_get(self._h, i, ctypes.byref(t), ctypes.byref(w), ctypes.byref(h),
                                           ctypes.byref(px), _ptr(verts, ctypes.c_float), _ptr(normal, ctypes.c_float),
                                           _ptr(focus, ctypes.c_float)))
        return {"type": t.value, "width": w.value, "height": h.value, "pixel_length": np.float32(px.value),
                "vertices": verts.reshape(4, 3), "normal": normal, "focus": focus}

    def heliostat(self, i: int) -> dict:
        t, g, nf, ns, sb = (ctypes.c_int() for _ in range(5))
        pos, size, normal = (np.zeros(3, np.float32) for _ in range(3))
        fl = ctypes.c_float()
        check(self._lib.qmcrt_heliostat_get(self._h, i, ctypes.byref(t), ctypes.byref(g), ctypes.byref(nf),
                                            ctypes.byref(ns), ctypes.byref(sb), _ptr(pos, ctypes.c_float),
                                            _ptr(size, ctypes.c_float), _ptr(normal, ctypes.c_float),
                                            ctypes.byref(fl)))
        return {"type": t.value, "grid": g.value, "num_facets": nf.value, "num_sub": ns.value,
                "sub_begin": sb.value, "pos": pos, "size": size, "normal": normal, "focus_length": np.float32(fl.value)}

    def grid(self, i: int) -> dict:
        cells = np.zeros(3, np.int32)
        nsub, nnz, recv, start, count = (ctypes.c_int() for _ in range(5))
        check(self._lib.qmcrt_grid_get(self._h, i, _ptr(cells, ctypes.c_int), ctypes.byref(nsub), ctypes.byref(nnz),
                                       ctypes.byref(recv), ctypes.byref(start), ctypes.byref(count)))
        n_cells = int(np.prod(cells))
        index = np.zeros(n_cells + 1, np.int32)
        match = np.zeros(max(nnz.value, 1), np.int32)
        check(self._lib.qmcrt_grid_csr(self._h, i, _ptr(index, ctypes.c_int), _ptr(match, ctypes.c_int)))
        verts = np.zeros((max(nsub.value, 1) * 3, 3), np.float32)
        check(self._lib.qmcrt_grid_vertices(self._h, i, _ptr(verts, ctypes.c_float)))
        return {"cells": tuple(int(c) for c in cells), "num_sub": nsub.value, "receiver": recv.value,
                "start": start.value, "count": count.value, "index": index, "match": match[: nnz.value],
                "vertices": verts[: nsub.value * 3]}

    def facets(self, i: int) -> tuple[np.ndarray, np.ndarray]:
        """Micro-facet centres and normals computed on the device."""
        n = self.heliostat(i)["num_facets"]
        o = np.zeros((max(n, 1), 3), np.float32)
        nn = np.zeros((max(n, 1), 3), np.float32)
        check(self._lib.qmcrt_heliostat_facets(self._h, i, _ptr(o, ctypes.c_float), _ptr(nn, ctypes.c_float)))
        return o[:n], nn[:n]

    # -- sampling -------------------------------------------------------------
    def set_sample_pool(self, dirs: np.ndarray, perturbations: np.ndarray) -> None:
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        p = np.ascontiguousarray(perturbations, np.float32).reshape(-1, 3)
        L = self.info.num_per_sunshape_group
        check(self._lib.qmcrt_set_sample_pool(self._h, d.ctypes.data, p.ctypes.data, d.shape[0] // L, L, 0))

    def generate_sample_pool(self, seed: int, sunshape: int = SUNSHAPE_BUIE, half_angle: float = 0.00465) -> None:
        check(self._lib.qmcrt_generate_sample_pool(self._h, int(seed) & 0xFFFFFFFF, int(sunshape), float(half_angle)))

    def get_sample_pool(self) -> tuple[np.ndarray, np.ndarray]:
        d = np.zeros((self.pool_size, 3), np.float32)
        p = np.zeros((self.pool_size, 3), np.float32)
        check(self._lib.qmcrt_get_sample_pool(self._h, _ptr(d, ctypes.c_float), _ptr(p, ctypes.c_float)))
        return d, p

    def set_facet_offsets(self, heliostat: int, offsets: np.ndarray) -> None:
        o = np.ascontiguousarray(offsets, np.int32)
        check(self._lib.qmcrt_set_facet_offsets(self._h, heliostat, _ptr(o, ctypes.c_int), o.size))

    def get_facet_offsets(self, heliostat: int) -> np.ndarray:
        n = self.heliostat(heliostat)["num_facets"] + 1
        o = np.zeros(n, np.int32)
        check(self._lib.qmcrt_get_facet_offsets(self._h, heliostat, _ptr(o, ctypes.c_int), n))
        return o

    def generate_facet_offsets(self, seed: int) -> None:
        check(self._lib.qmcrt_generate_facet_offsets(self._h, int(seed) & 0xFFFFFFFF))

    def set_math_mode(self, exact) -> None:
        """True/1: exact build; False/0: production build; 2: production, 48 registers."""
        mode = int(exact) if not isinstance(exact, bool) else (1 if exact else 0)
        check(self._lib.qmcrt_set_math_mode(self._h, mode))

    def set_light_range(self, begin: int, end: int) -> None:
        check(self._lib.qmcrt_set_light_range(self._h, begin, end))

    # -- tracing --------------------------------------------------------------
    def trace(self, heliostats, stream=None) -> None:
        ids = np.ascontiguousarray(np.atleast_1d(np.asarray(heliostats, np.int32)))
        check(self._lib.qmcrt_trace_heliostats(self._h, _ptr(ids, ctypes.c_int), ids.size, _stream_handle(stream)))

    def image(self, receiver: int = 0) -> np.ndarray:
        w, h = ctypes.c_int(), ctypes.c_int()
        check(self._lib.qmcrt_receiver_image(self._h, receiver, None, ctypes.byref(w), ctypes.byref(h)))
        out = np.zeros((h.value, w.value), np.float32)
        check(self._lib.qmcrt_receiver_image(self._h, receiver, _ptr(out, ctypes.c_float), ctypes.byref(w),
                                             ctypes.byref(h)))
        return out

    def device_image(self, receiver: int = 0) -> tuple[int, int, int]:
        p = ctypes.c_void_p()
        w, h = ctypes.c_int(), ctypes.c_int()
        check(self._lib.qmcrt_receiver_device_image(self._h, receiver, ctypes.byref(p), ctypes.byref(w),
                                                    ctypes.byref(h)))
        return p.value, w.value, h.value

    def clear(self, receiver: int | None = None, stream=None) -> None:
        targets = range(self.num_receivers) if receiver is None else [receiver]
        for r in targets:
            check(self._lib.qmcrt_receiver_clear(self._h, r, _stream_handle(stream)))

    def power(self) -> tuple[np.ndarray, float]:
        per = np.zeros(self.num_heliostats, np.float64)
        total = ctypes.c_double()
        check(self._lib.qmcrt_power_fp64(self._h, _ptr(per, ctypes.c_double), ctypes.byref(total)))
        return per, total.value

    def clear_power(self) -> None:
        check(self._lib.qmcrt_power_clear(self._h))

    def diagnostics(self) -> dict:
        out = (ctypes.c_ulonglong * 4)()
        check(self._lib.qmcrt_diagnostics(self._h, out))
        return {"clamped": out[0], "walk_capped": out[1]}

    def hit_records(self, heliostat: int, facet_begin: int, facet_end: int, light_begin: int,
                    light_end: int) -> np.ndarray:
        n = (facet_end - facet_begin) * (light_end - light_begin)
        out = np.zeros(max(n, 1), np.int32)
        check(self._lib.qmcrt_debug_hit_records(self._h, heliostat, facet_begin, facet_end, light_begin, light_end,
                                                _ptr(out, ctypes.c_int)))
        return out[:n]

    def load_tasks(self, path) -> tuple[list, list, bool]:
        cap = self.num_heliostats + 1
        hs = np.zeros(cap, np.int32)
        rs = np.zeros(cap, np.int32)
        nh, nr, st = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.qmcrt_load_tasks(self._h, str(path).encode(), _ptr(hs, ctypes.c_int), ctypes.byref(nh), cap,
                                         _ptr(rs, ctypes.c_int), ctypes.byref(nr), ctypes.byref(st)))
        return hs[: nh.value].tolist(), rs[: nr.value].tolist(), bool(st.value)


def smooth_device(device_ptr: int, width: int, height: int, radius: int, ratio: float, stream=None) -> None:
    """In-place trimmed mean of a device image (qmcrt_smooth)."""
    check(load().qmcrt_smooth(ctypes.c_void_p(device_ptr), width, height, radius, float(ratio),
                              _stream_handle(stream)))


def save_text(path, data: np.ndarray, precision: int = 2) -> float:
    a = np.ascontiguousarray(data, np.float32)
    mx = ctypes.c_float()
    check(load().qmcrt_save_text(str(path).encode(), a.shape[0], a.shape[1], _ptr(a, ctypes.c_float), precision,
                                 ctypes.byref(mx)))
    return mx.value


def pipeline_run(argv: list[str]) -> int:
    arr = (ctypes.c_char_p * (len(argv) + 1))(*[a.encode() for a in argv], None)
    return load().qmcrt_pipeline_run(len(argv), arr)


# ---- reference-named facade ------------------------------------------------
class QuasiMonteCarloRayTracer:
    """QuasiMonteCarloRayTracer (QuasiMonteCarloRayTracing/QuasiMonteCarloRayTracer.h:11-28)."""

    def rayTracing(self, scene: Scene, heliostat_id: int, stream=None) -> None:  # noqa: N802
        scene.trace([heliostat_id], stream)


class ImageSmoother:
    """ImageSmoother::image_smooth (Tool/Smoother/ImageSmoother.cuh:18-22)."""

    @staticmethod
    def image_smooth(device_ptr: int, kernel_radius: int, trimmed_ratio: float, width: int, height: int,
                     stream=None) -> None:
        smooth_device(device_ptr, width, height, kernel_radius, trimmed_ratio, stream)


class ImageSaver:
    """ImageSaver::saveText (Tool/ImageSaver/ImageSaver.h:10-13)."""

    @staticmethod
    def saveText(filename, height: int, width: int, h_data: np.ndarray, precision: int = 2) -> float:  # noqa: N802
        return save_text(filename, np.asarray(h_data, np.float32).reshape(height, width), precision)


class RayTracingPipeline:
    """RayTracingPipeline::rayTracing(argc, argv) (RayTracingPipeline/RayTracingPipeline.h:11-17)."""

    @staticmethod
    def rayTracing(argv: list[str]) -> int:  # noqa: N802
        return pipeline_run(argv)


def executable() -> Path:
    return Path(__file__).resolve().parent / "bin" / "qmcrt"
