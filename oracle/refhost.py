"""CPU ORACLE - test infrastructure only: ctypes harness for oracle/_ref/libref_host.so.

The library is the reference's own host code (see build_ref.py).  Its scene
state lives in the reference's SolarScene / SceneConfiguration singletons,
so one scene is loaded at a time per process.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libref_host.so"

_i = ctypes.c_int
_f = ctypes.c_float
_pi = ctypes.POINTER(ctypes.c_int)
_pf = ctypes.POINTER(ctypes.c_float)
_pd = ctypes.POINTER(ctypes.c_double)
_pll = ctypes.POINTER(ctypes.c_longlong)


class RefTraceArgs(ctypes.Structure):
    _fields_ = [
        ("ids", _pi), ("n_ids", _i), ("pool_dirs", _pf), ("pool_pert", _pf), ("pool_size", _i),
        ("offsets", _pi), ("offset_base", _pll), ("light_begin", _i), ("light_end", _i),
        ("facet_stride", _i), ("facet_phase", _i), ("images", _pd), ("image_base", _pll), ("power", _pd),
        ("counters", _pll), ("rec_id", _i), ("rec_facet_begin", _i), ("rec_facet_end", _i), ("records", _pi),
        ("threads", _i),
    ]


_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(str(LIB))
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_load_config.argtypes = [ctypes.c_char_p]
        L.ref_read_scene.argtypes = [ctypes.c_char_p]
        L.ref_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _pi]
        L.ref_receiver.argtypes = [_i, _pi, _pf]
        L.ref_heliostat.argtypes = [_i, _pi, _pf]
        L.ref_grid.argtypes = [_i, _pi]
        L.ref_grid_csr.argtypes = [_i, _pi, _pi]
        L.ref_grid_vertices.argtypes = [_i, _pf]
        L.ref_facets.argtypes = [_i, _pf, _pf]
        L.ref_collision.argtypes = [_i, _pf, _pf]
        L.ref_receiver_hit.argtypes = [_i, _pf, _pf, _pf]
        L.ref_trace.argtypes = [ctypes.POINTER(RefTraceArgs)]
        L.ref_smooth.argtypes = [_pf, _pf, _i, _i, _i, _f]
        L.ref_buie_table.argtypes = [_f, _i, _pf, _pf, _pf, _pf]
        L.ref_buie_theta.argtypes = [_f, _i, _pf, _pf, _i]
        L.ref_load_tasks.argtypes = [ctypes.c_char_p, _pi, _pi, _pi, _pi]
        L.ref_save_text.argtypes = [ctypes.c_char_p, _i, _i, _pf]
        L.ref_save_text.restype = _f
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def load_config(path) -> int:
    return lib().ref_load_config(str(path).encode())


def read_scene(path) -> bool:
    return bool(lib().ref_read_scene(str(path).encode()))


class RefScene:
    """The reference's SolarScene after SceneFileRead + the geometry half of processScene."""

    def __init__(self, scene_path, config_path, lights_per_group: int | None = None):
        c = np.zeros(3, np.int32)
        rc = lib().ref_load(str(scene_path).encode(), str(config_path).encode(), _p(c, _i))
        if rc != 0:
            raise RuntimeError(f"reference failed to load the scene ({rc})")
        self.num_receivers, self.num_grids, self.num_heliostats = map(int, c)

    def receiver(self, i):
        ints = np.zeros(3, np.int32)
        vals = np.zeros(19, np.float32)
        lib().ref_receiver(i, _p(ints, _i), _p(vals, _f))
        return {"type": int(ints[0]), "width": int(ints[1]), "height": int(ints[2]), "pixel_length": vals[0],
                "vertices": vals[1:13].reshape(4, 3), "normal": vals[13:16], "focus": vals[16:19]}

    def heliostat(self, i):
        ints = np.zeros(5, np.int32)
        vals = np.zeros(4, np.float32)
        lib().ref_heliostat(i, _p(ints, _i), _p(vals, _f))
        return {"type": int(ints[0]), "grid": int(ints[1]), "num_facets": int(ints[2]), "num_sub": int(ints[3]),
                "sub_begin": int(ints[4]), "normal": vals[0:3], "focus_length": vals[3]}

    def grid(self, i):
        ints = np.zeros(5, np.int32)
        lib().ref_grid(i, _p(ints, _i))
        cells = tuple(int(x) for x in ints[:3])
        nnz, nsub = int(ints[3]), int(ints[4])
        index = np.zeros(cells[0] * cells[1] * cells[2] + 1, np.int32)
        match = np.zeros(max(nnz, 1), np.int32)
        lib().ref_grid_csr(i, _p(index, _i), _p(match, _i))
        verts = np.zeros((max(nsub, 1) * 3, 3), np.float32)
        lib().ref_grid_vertices(i, _p(verts, _f))
        return {"cells": cells, "index": index, "match": match[:nnz], "vertices": verts[: nsub * 3]}

    def facets(self, i):
        n = self.heliostat(i)["num_facets"]
        o = np.zeros((max(n, 1), 3), np.float32)
        nn = np.zeros((max(n, 1), 3), np.float32)
        lib().ref_facets(i, _p(o, _f), _p(nn, _f))
        return o[:n], nn[:n]

    def collision(self, heliostat, origin, direction) -> bool:
        o = np.asarray(origin, np.float32)
        d = np.asarray(direction, np.float32)
        return bool(lib().ref_collision(heliostat, _p(o, _f), _p(d, _f)))

    def receiver_hit(self, recv, origin, direction):
        o = np.asarray(origin, np.float32)
        d = np.asarray(direction, np.float32)
        tuv = np.zeros(3, np.float32)
        hit = lib().ref_receiver_hit(recv, _p(o, _f), _p(d, _f), _p(tuv, _f))
        return bool(hit), tuv

    def trace(self, ids, pool_dirs, pool_pert, offsets, per_group, light_begin=0, light_end=None, facet_stride=1,
              facet_phase=0, images=True, record=None, threads=0):
        ids = np.ascontiguousarray(np.array(ids, np.int32))
        dirs = np.ascontiguousarray(np.asarray(pool_dirs, np.float32).reshape(-1, 3))
        pert = np.ascontiguousarray(np.asarray(pool_pert, np.float32).reshape(-1, 3))
        P = dirs.shape[0]
        nf = [self.heliostat(i)["num_facets"] for i in range(self.num_heliostats)]
        base = np.zeros(self.num_heliostats, np.int64)
        chunks, pos = [], 0
        for h in range(self.num_heliostats):
            base[h] = pos
            o = np.asarray(offsets[h], np.int32) if h in offsets else np.zeros(nf[h] + 1, np.int32)
            chunks.append(o)
            pos += o.size
        offs = np.ascontiguousarray(np.concatenate(chunks).astype(np.int32))
        recs = [self.receiver(r) for r in range(self.num_receivers)]
        img_base = np.zeros(self.num_receivers + 1, np.int64)
        for r, rc in enumerate(recs):
            img_base[r + 1] = img_base[r] + rc["width"] * rc["height"]
        img = np.zeros(max(int(img_base[-1]), 1), np.float64)
        power = np.zeros(self.num_heliostats, np.float64)
        counters = np.zeros(6, np.int64)
        le = per_group if light_end is None else light_end
        a = RefTraceArgs()
        a.ids, a.n_ids = _p(ids, _i), ids.size
        a.pool_dirs, a.pool_pert, a.pool_size = _p(dirs, _f), _p(pert, _f), P
        a.offsets, a.offset_base = _p(offs, _i), _p(base, ctypes.c_longlong)
        a.light_begin, a.light_end = light_begin, le
        a.facet_stride, a.facet_phase = facet_stride, facet_phase
        a.images = _p(img, ctypes.c_double) if images else None
        a.image_base = _p(img_base, ctypes.c_longlong)
        a.power = _p(power, ctypes.c_double)
        a.counters = _p(counters, ctypes.c_longlong)
        rec = None
        if record is not None:
            rid, fb, fe = record
            rec = np.full((fe - fb) * (le - light_begin), -4, np.int32)
            a.rec_id, a.rec_facet_begin, a.rec_facet_end, a.records = rid, fb, fe, _p(rec, _i)
        else:
            a.rec_id, a.rec_facet_begin, a.rec_facet_end, a.records = -1, 0, 0, None
        a.threads = threads
        lib().ref_trace(ctypes.byref(a))
        out = [img[img_base[r]:img_base[r + 1]].reshape(rc["height"], rc["width"]).copy() for r, rc in enumerate(recs)]
        names = ["rays", "shadowed", "blocked", "missed", "hit", "clamped"]
        return {"images": out, "power": power, "counters": dict(zip(names, map(int, counters))), "records": rec}

    def load_tasks(self, path):
        n = self.num_heliostats + 1
        ids = np.zeros(n, np.int32)
        grids = np.zeros(n, np.int32)
        ni, ng = ctypes.c_int(), ctypes.c_int()
        rc = lib().ref_load_tasks(str(path).encode(), _p(ids, _i), ctypes.byref(ni), _p(grids, _i), ctypes.byref(ng))
        if rc < 0:
            raise ValueError(lib().ref_last_error().decode())
        return sorted(ids[: ni.value].tolist()), sorted(grids[: ng.value].tolist()), bool(rc)


def smooth(image, radius, ratio):
    img = np.ascontiguousarray(image, np.float32)
    out = np.zeros_like(img)
    h, w = img.shape
    lib().ref_smooth(_p(img, _f), _p(out, _f), w, h, radius, ratio)
    return out


def buie_table(csr, groups):
    cx = np.zeros(groups + 1, np.float32)
    cy = np.zeros(groups + 1, np.float32)
    k = np.zeros(groups, np.float32)
    sc = np.zeros(5, np.float32)
    lib().ref_buie_table(csr, groups, _p(cx, _f), _p(cy, _f), _p(k, _f), _p(sc, _f))
    return {"cdf_x": cx, "cdf_y": cy, "k": k, "less_465": sc[0], "gamma": sc[1], "A": sc[2], "B": sc[3], "C": sc[4]}


def buie_theta(csr, groups, uniforms):
    u = np.ascontiguousarray(uniforms, np.float32)
    out = np.zeros_like(u)
    lib().ref_buie_theta(csr, groups, _p(u, _f), _p(out, _f), u.size)
    return out


def save_text(path, data) -> float:
    a = np.ascontiguousarray(data, np.float32)
    return lib().ref_save_text(str(path).encode(), a.shape[0], a.shape[1], _p(a, _f))
