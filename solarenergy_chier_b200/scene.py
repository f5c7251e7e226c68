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
        """True/1: exact build; False/0: production build; 2: production, 64 registers (4 blocks/SM);
        3: production with approximate per-ray arithmetic after the shadow test;
        4: production with approximate arithmetic after the receiver's decisions."""
        mode = int(exact) if not isinstance(exact, bool) else (1 if exact else 0)
        check(self._lib.qmcrt_set_math_mode(self._h, mode))

    def set_light_range(self, begin: int, end: int) -> None:
        check(self._lib.qmcrt_set_light_range(self._h, begin, end))

    def set_launch_shape(self, shape: int) -> None:
        """Launch shape of the production build's flux launches (launch_shapes())."""
        check(self._lib.qmcrt_set_launch_shape(self._h, int(shape)))

    def autotune(self, heliostats, stream=None) -> tuple[int, list]:
        """Times every launch shape on `heliostats` at the current light range and
        keeps the fastest: (chosen shape, ms per shape).  Clears images and powers."""
        ids = np.ascontiguousarray(np.atleast_1d(np.asarray(heliostats, np.int32)))
        best = ctypes.c_int()
        table = (ctypes.c_float * 16)()
        check(self._lib.qmcrt_autotune(self._h, _ptr(ids, ctypes.c_int), ids.size, _stream_handle(stream),
                                       ctypes.byref(best), table))
        return best.value, list(table[: len(launch_shapes())])

    def shadow_free(self) -> np.ndarray:
        """Per heliostat: 1 shadow walks skipped, k + 1 only k listed candidate
        shadowing heliostats (rays missing their boxes skip the walk), 0 walk."""
        f = np.zeros(self.num_heliostats, np.int32)
        check(self._lib.qmcrt_debug_shadow_free(self._h, _ptr(f, ctypes.c_int)))
        return f

    def block_free(self, grid: int = 0) -> np.ndarray:
        """Per sub-heliostat of a grid: 1 block walks skipped, k + 1 only k listed
        candidate blockers (rays missing their boxes skip the walk), 0 walk."""
        f = np.zeros(max(self.grid(grid)["num_sub"], 1), np.int32)
        check(self._lib.qmcrt_debug_block_free(self._h, grid, _ptr(f, ctypes.c_int)))
        return f

    def build_grid_on_device(self, grid: int = 0) -> float:
        """Rebuild the grid's device cell lists on the GPU; returns the build's device ms."""
        ms = ctypes.c_float()
        check(self._lib.qmcrt_grid_build_device(self._h, grid, ctypes.byref(ms)))
        return ms.value

    def device_grid_cells(self, grid: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """(ranges (cells, 2), entries (n, 4)) of the grid's device cell lists."""
        n = ctypes.c_longlong()
        check(self._lib.qmcrt_debug_grid_cells(self._h, grid, None, None, ctypes.byref(n)))
        c = self.grid(grid)["cells"]
        ranges = np.zeros((int(np.prod(c)), 2), np.int32)
        entries = np.zeros((max(n.value, 1), 4), np.int32)
        check(self._lib.qmcrt_debug_grid_cells(self._h, grid, _ptr(ranges, ctypes.c_int), _ptr(entries, ctypes.c_int),
                                               ctypes.byref(n)))
        return ranges, entries[:n.value]

    def set_sun(self, sun_dir) -> None:
        """Re-orient the field toward a new sun direction (direction of travel)."""
        d = np.ascontiguousarray(np.asarray(sun_dir, np.float32).reshape(3))
        check(self._lib.qmcrt_scene_set_sun(self._h, _ptr(d, ctypes.c_float)))

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

    def hit_bit_words(self, heliostats) -> int:
        """32-bit words of the per-ray hit bits of `heliostats` over the light range."""
        ids = np.ascontiguousarray(np.atleast_1d(np.asarray(heliostats, np.int32)))
        words = ctypes.c_longlong()
        check(self._lib.qmcrt_debug_hit_bits(self._h, _ptr(ids, ctypes.c_int), ids.size, None, 0,
                                             ctypes.byref(words), None))
        return words.value

    def hit_bits(self, heliostats, device_ptr: int, capacity_words: int, stream=None) -> int:
        """One hit bit per ray of `heliostats` (current light range and math
        mode, nothing deposited) into `capacity_words` 32-bit words of device
        memory at `device_ptr`; returns the words written."""
        ids = np.ascontiguousarray(np.atleast_1d(np.asarray(heliostats, np.int32)))
        words = ctypes.c_longlong()
        check(self._lib.qmcrt_debug_hit_bits(self._h, _ptr(ids, ctypes.c_int), ids.size, ctypes.c_void_p(device_ptr),
                                             capacity_words, ctypes.byref(words), _stream_handle(stream)))
        return words.value

    def load_tasks(self, path) -> tuple[list, list, bool]:
        cap = self.num_heliostats + 1
        hs = np.zeros(cap, np.int32)
        rs = np.zeros(cap, np.int32)
        nh, nr, st = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.qmcrt_load_tasks(self._h, str(path).encode(), _ptr(hs, ctypes.c_int), ctypes.byref(nh), cap,
                                         _ptr(rs, ctypes.c_int), ctypes.byref(nr), ctypes.byref(st)))
        return hs[: nh.value].tolist(), rs[: nr.value].tolist(), bool(st.value)


class Batch:
    """Many (scene, sun) instances traced by one launch (qmcrt_batch_*).

    `scenes` is a list of loaded Scenes on one device; `instances` a list of
    (scene index, sun direction) pairs.  Every instance has its own images and
    FP64 powers; the sun-dependent geometry is prepared on the GPU."""

    def __init__(self, scenes, instances):
        lib = load()
        self._lib = lib
        self._scenes = list(scenes)  # keep the scenes alive as long as the batch
        hs = (ctypes.c_void_p * len(self._scenes))(*[s.handle.value for s in self._scenes])
        idx = np.ascontiguousarray(np.array([int(k) for k, _ in instances], np.int32))
        suns = np.ascontiguousarray(np.array([np.asarray(d, np.float32) for _, d in instances], np.float32).reshape(-1, 3))
        self._instances = [(int(k), suns[i]) for i, (k, _) in enumerate(instances)]
        handle = ctypes.c_void_p()
        check(lib.qmcrt_batch_create(hs, len(self._scenes), _ptr(idx, ctypes.c_int), _ptr(suns, ctypes.c_float),
                                     len(self._instances), ctypes.byref(handle)))
        self._h = handle

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.qmcrt_batch_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_instances(self) -> int:
        return len(self._instances)

    def info(self) -> dict:
        n, t, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        check(self._lib.qmcrt_batch_info(self._h, ctypes.byref(n), ctypes.byref(t), ctypes.byref(r)))
        return {"instances": n.value, "tasks": t.value, "rays_per_trace": r.value}

    def set_suns(self, sun_dirs, stream=None) -> None:
        d = np.ascontiguousarray(np.asarray(sun_dirs, np.float32).reshape(-1, 3))
        if d.shape[0] != self.num_instances:
            raise ValueError("one sun direction per instance")
        check(self._lib.qmcrt_batch_set_suns(self._h, _ptr(d, ctypes.c_float), _stream_handle(stream)))

    def set_light_range(self, begin: int, end: int) -> None:
        check(self._lib.qmcrt_batch_set_light_range(self._h, begin, end))

    def set_math_mode(self, mode) -> None:
        check(self._lib.qmcrt_batch_set_math_mode(self._h, int(mode)))

    def trace(self, stream=None) -> None:
        check(self._lib.qmcrt_batch_trace(self._h, _stream_handle(stream)))

    def capture_graph(self, clear_first: bool = True) -> None:
        check(self._lib.qmcrt_batch_capture_graph(self._h, int(bool(clear_first))))

    def graph_launch(self, stream=None) -> None:
        check(self._lib.qmcrt_batch_graph_launch(self._h, _stream_handle(stream)))

    def clear(self, stream=None) -> None:
        check(self._lib.qmcrt_batch_clear(self._h, _stream_handle(stream)))

    def autotune(self, stream=None) -> tuple[int, list]:
        """Times every launch shape of the production build on this batch and
        keeps the fastest: (chosen shape, ms per shape)."""
        m = ctypes.c_int()
        table = (ctypes.c_float * 16)()
        check(self._lib.qmcrt_batch_autotune_shapes(self._h, _stream_handle(stream), ctypes.byref(m), table))
        return m.value, list(table[: len(launch_shapes())])

    def set_launch_shape(self, shape: int) -> None:
        check(self._lib.qmcrt_batch_set_launch_shape(self._h, int(shape)))

    def image(self, instance: int, receiver: int = 0) -> np.ndarray:
        w, h = ctypes.c_int(), ctypes.c_int()
        check(self._lib.qmcrt_batch_image(self._h, instance, receiver, None, ctypes.byref(w), ctypes.byref(h)))
        out = np.zeros((h.value, w.value), np.float32)
        check(self._lib.qmcrt_batch_image(self._h, instance, receiver, _ptr(out, ctypes.c_float), ctypes.byref(w),
                                          ctypes.byref(h)))
        return out

    def geometry(self, instance: int, grid: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """Device-prepared sub-heliostat vertices of one grid and heliostat normals."""
        s = self._scenes[self._instances[instance][0]]
        g = s.grid(grid)
        verts = np.zeros((g["num_sub"] * 3, 3), np.float32)
        normals = np.zeros((s.num_heliostats, 3), np.float32)
        check(self._lib.qmcrt_batch_debug_geometry(self._h, instance, grid, _ptr(verts, ctypes.c_float),
                                                   _ptr(normals, ctypes.c_float)))
        return verts, normals

    def power(self, instance: int) -> tuple[np.ndarray, float]:
        k = self._instances[instance][0]
        per = np.zeros(self._scenes[k].num_heliostats, np.float64)
        total = ctypes.c_double()
        check(self._lib.qmcrt_batch_power_fp64(self._h, instance, _ptr(per, ctypes.c_double), ctypes.byref(total)))
        return per, total.value


class Diff:
    """Differentiable forward / adjoint over one scene (qmcrt_diff_*, qmcrt_fwd, qmcrt_bwd).

    Parameters per heliostat: aim offset (du, dv) in metres and normal offset
    (a, b) in radians; `forward()` returns the loss against the target flux,
    `backward()` its gradient, shape (num_heliostats, 4)."""

    def __init__(self, scene: Scene, sigma_px: float = 2.0, suns=None):
        """suns: None for the scene's own sun, else sun directions (n, 3): one
        pair over all of them, parameters shared, receiver index k * R + r."""
        self._lib = load()
        self._scene = scene  # the scene must outlive the pair
        h = ctypes.c_void_p()
        if suns is None:
            check(self._lib.qmcrt_diff_create(scene.handle, float(sigma_px), ctypes.byref(h)))
            self.num_suns = 1
        else:
            d = np.ascontiguousarray(np.asarray(suns, np.float32).reshape(-1, 3))
            check(self._lib.qmcrt_diff_create_suns(scene.handle, _ptr(d, ctypes.c_float), d.shape[0],
                                                   float(sigma_px), ctypes.byref(h)))
            self.num_suns = d.shape[0]
        self._h = h
        self.num_heliostats = scene.num_heliostats

    def set_hit_records(self, mode: int, segment_rays: int = 0) -> None:
        """0 automatic, 1 checkpoint, 2 recompute (segment_rays per segment; 0 keeps it)."""
        check(self._lib.qmcrt_diff_set_hit_records(self._h, int(mode), int(segment_rays)))

    def hit_records(self) -> tuple[bool, int]:
        """(recomputed, checkpoint bytes) of the last forward."""
        r, n = ctypes.c_int(), ctypes.c_longlong()
        check(self._lib.qmcrt_diff_hit_records(self._h, ctypes.byref(r), ctypes.byref(n)))
        return bool(r.value), n.value

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.qmcrt_diff_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, aim=None, normal=None) -> None:
        def arr(x):
            if x is None:
                return None, None
            a = np.ascontiguousarray(np.asarray(x, np.float32).reshape(self.num_heliostats, 2))
            return a, _ptr(a, ctypes.c_float)

        a, pa = arr(aim)
        n, pn = arr(normal)
        check(self._lib.qmcrt_diff_set_params(self._h, pa, pn))

    def set_target(self, target: np.ndarray, receiver: int = 0) -> None:
        w, h = ctypes.c_int(), ctypes.c_int()
        check(self._lib.qmcrt_diff_flux(self._h, receiver, None, ctypes.byref(w), ctypes.byref(h)))
        t = np.ascontiguousarray(np.asarray(target, np.float32))
        if t.shape != (h.value, w.value):
            raise ValueError(f"target shape {t.shape} != receiver image ({h.value}, {w.value})")
        check(self._lib.qmcrt_diff_set_target(self._h, receiver, _ptr(t, ctypes.c_float)))

    def set_light_range(self, begin: int, end: int) -> None:
        check(self._lib.qmcrt_diff_set_light_range(self._h, begin, end))

    def forward(self, stream=None) -> float:
        loss = ctypes.c_double()
        check(self._lib.qmcrt_fwd(self._h, ctypes.byref(loss), _stream_handle(stream)))
        return loss.value

    def backward(self, stream=None) -> np.ndarray:
        g = np.zeros((self.num_heliostats, 4), np.float64)
        check(self._lib.qmcrt_bwd(self._h, _ptr(g, ctypes.c_double), _stream_handle(stream)))
        return g

    def flux(self, receiver: int = 0) -> np.ndarray:
        w, h = ctypes.c_int(), ctypes.c_int()
        check(self._lib.qmcrt_diff_flux(self._h, receiver, None, ctypes.byref(w), ctypes.byref(h)))
        out = np.zeros((h.value, w.value), np.float32)
        check(self._lib.qmcrt_diff_flux(self._h, receiver, _ptr(out, ctypes.c_float), ctypes.byref(w), ctypes.byref(h)))
        return out

    def plain(self, stream=None) -> None:
        """Trace the current parameters with the plain tracer (nearest-pixel flux)."""
        check(self._lib.qmcrt_diff_plain(self._h, _stream_handle(stream)))

    def image(self, receiver: int = 0) -> np.ndarray:
        """Unsmoothed flux of the last trace (forward: bilinear deposit; plain: binned)."""
        w, h = ctypes.c_int(), ctypes.c_int()
        check(self._lib.qmcrt_diff_image(self._h, receiver, None, ctypes.byref(w), ctypes.byref(h)))
        out = np.zeros((h.value, w.value), np.float32)
        check(self._lib.qmcrt_diff_image(self._h, receiver, _ptr(out, ctypes.c_float), ctypes.byref(w),
                                         ctypes.byref(h)))
        return out

    def power(self) -> tuple[np.ndarray, float]:
        """FP64 per-heliostat powers and total of the last trace."""
        per = np.zeros(self.num_heliostats, np.float64)
        total = ctypes.c_double()
        check(self._lib.qmcrt_diff_power(self._h, _ptr(per, ctypes.c_double), ctypes.byref(total)))
        return per, total.value


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


def launch_shapes() -> list[tuple[int, int, bool]]:
    """(threads per block, warp-chunk iterations, persistent) of each launch shape of the production build."""
    lib = load()
    n = ctypes.c_int()
    check(lib.qmcrt_launch_shapes(None, None, None, ctypes.byref(n)))
    t = np.zeros(n.value, np.int32)
    c = np.zeros(n.value, np.int32)
    ps = np.zeros(n.value, np.int32)
    check(lib.qmcrt_launch_shapes(_ptr(t, ctypes.c_int), _ptr(c, ctypes.c_int), _ptr(ps, ctypes.c_int),
                                  ctypes.byref(n)))
    return [(a, b, bool(x)) for a, b, x in zip(t.tolist(), c.tolist(), ps.tolist())]


def executable() -> Path:
    return Path(__file__).resolve().parent / "bin" / "qmcrt"
