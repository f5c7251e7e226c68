"""CPU ORACLE - test infrastructure only: ctypes harness for qmcrt_oracle.cpp.

Only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and
`--impl reference`) import this module, as the checker.  The product package
never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

from . import scene_text

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
SRC = HERE / "qmcrt_oracle.cpp"

_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
_pi = ctypes.POINTER(ctypes.c_int)
_pf = ctypes.POINTER(ctypes.c_float)
_pd = ctypes.POINTER(ctypes.c_double)
_pll = ctypes.POINTER(ctypes.c_longlong)
_pu = ctypes.POINTER(ctypes.c_uint32)


class Desc(ctypes.Structure):
    _fields_ = [
        ("sun_dir", _f * 3), ("dni", _f), ("csr", _f), ("recv_px", _f), ("helio_px", _f), ("rho", _f), ("sigma", _f),
        ("groups", _i), ("per_group", _i), ("its_groups", _i),
        ("n_recv", _i), ("recv_type", _pi), ("recv_pos", _pf), ("recv_size", _pf), ("recv_norm", _pf), ("recv_face", _pi),
        ("n_grid", _i), ("grid_type", _pi), ("grid_pos", _pf), ("grid_size", _pf), ("grid_inter", _pf),
        ("grid_n", _pi), ("grid_htype", _pi), ("grid_start", _pi), ("grid_recv", _pi),
        ("n_helio", _i), ("h_type", _pi), ("h_pos", _pf), ("h_size", _pf), ("h_gap", _pf), ("h_matrix", _pi),
        ("h_surface", _pf), ("h_grid", _pi), ("h_local_off", _pi), ("local_centers", _pf), ("local_normals", _pf),
    ]


class TraceArgs(ctypes.Structure):
    _fields_ = [
        ("ids", _pi), ("n_ids", _i), ("pool_dirs", _pf), ("pool_pert", _pf), ("pool_size", _i),
        ("offsets", _pi), ("offset_base", _pll), ("light_begin", _i), ("light_end", _i),
        ("facet_stride", _i), ("facet_phase", _i), ("images", _pd), ("image_base", _pll), ("power", _pd),
        ("counters", _pll), ("rec_id", _i), ("rec_facet_begin", _i), ("rec_facet_end", _i), ("records", _pi),
        ("threads", _i), ("record_only", _i),
    ]


def build(force: bool = False) -> Path:
    """Compile the oracle with g++ (no CUDA)."""
    LIB.parent.mkdir(exist_ok=True)
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fopenmp", "-o", str(LIB), str(SRC)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.POINTER(Desc), _i]
        L.oracle_free.argtypes = [ctypes.c_void_p]
        L.oracle_counts.argtypes = [ctypes.c_void_p, _pi]
        L.oracle_receiver.argtypes = [ctypes.c_void_p, _i, _pi, _pd]
        L.oracle_heliostat.argtypes = [ctypes.c_void_p, _i, _pi, _pd]
        L.oracle_grid.argtypes = [ctypes.c_void_p, _i, _pi]
        L.oracle_grid_csr.argtypes = [ctypes.c_void_p, _i, _pi, _pi]
        L.oracle_grid_vertices.argtypes = [ctypes.c_void_p, _i, _pd]
        L.oracle_facets.argtypes = [ctypes.c_void_p, _i, _pd, _pd]
        L.oracle_trace.argtypes = [ctypes.c_void_p, ctypes.POINTER(TraceArgs)]
        L.oracle_walk.argtypes = [ctypes.c_void_p, _i, _i, _i, _pd, _pd]
        L.oracle_walk.restype = _i
        L.oracle_receiver_hit.argtypes = [ctypes.c_void_p, _i, _pf, _pf, _pf]
        L.oracle_receiver_hit.restype = _i
        L.oracle_smooth.argtypes = [_pf, _pf, _i, _i, _i, _f]
        L.oracle_buie.argtypes = [_f, _i, _pf, _pf, _i]
        L.oracle_buie_table.argtypes = [_f, _i, _pf, _pf, _pf, _pf]
        L.oracle_sobol2.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _i, _pu]
        L.oracle_facet_offsets.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _i, ctypes.c_uint32, _pi]
        L.oracle_mix32.argtypes = [ctypes.c_uint32]
        L.oracle_mix32.restype = ctypes.c_uint32
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


class OracleScene:
    """A processed scene held by the C++ oracle in float (32) or double (64)."""

    def __init__(self, scene: scene_text.SceneText, config: dict, precision: int = 32):
        self.scene = scene
        self.config = config
        self._keep = []
        d = Desc()
        d.sun_dir = (_f * 3)(*[float(x) for x in config["sun_dir"]])
        d.dni = config["dni"]
        d.csr = config["csr"]
        d.recv_px = config["receiver_pixel_length"]
        d.helio_px = config["helio_pixel_length"]
        d.rho = config["helio_reflected_rate"]
        d.sigma = config["helio_disturb_std"]
        d.groups = config["num_of_sunshape_groups"]
        d.per_group = config["num_per_sunshape_group"]
        d.its_groups = config["inverse_transform_sampling_groups"]
        R, G, H = scene.receivers, scene.grids, scene.heliostats

        def arr(values, dtype):
            a = np.ascontiguousarray(np.array(values, dtype=dtype))
            if a.size == 0:
                a = np.zeros(1, dtype)
            self._keep.append(a)
            return a

        d.n_recv = len(R)
        d.recv_type = _p(arr([r.type for r in R], np.int32), _i)
        d.recv_pos = _p(arr([r.pos for r in R], np.float32), _f)
        d.recv_size = _p(arr([r.size for r in R], np.float32), _f)
        d.recv_norm = _p(arr([r.norm for r in R], np.float32), _f)
        d.recv_face = _p(arr([r.face for r in R], np.int32), _i)
        d.n_grid = len(G)
        d.grid_type = _p(arr([g.type for g in G], np.int32), _i)
        d.grid_pos = _p(arr([g.pos for g in G], np.float32), _f)
        d.grid_size = _p(arr([g.size for g in G], np.float32), _f)
        d.grid_inter = _p(arr([g.inter for g in G], np.float32), _f)
        d.grid_n = _p(arr([g.n for g in G], np.int32), _i)
        d.grid_htype = _p(arr([g.helio_type for g in G], np.int32), _i)
        d.grid_start = _p(arr([g.start for g in G], np.int32), _i)
        d.grid_recv = _p(arr([g.receiver for g in G], np.int32), _i)
        d.n_helio = len(H)
        d.h_type = _p(arr([h.type for h in H], np.int32), _i)
        d.h_pos = _p(arr([h.pos for h in H], np.float32), _f)
        d.h_size = _p(arr([h.size for h in H], np.float32), _f)
        d.h_gap = _p(arr([h.gap for h in H], np.float32), _f)
        d.h_matrix = _p(arr([h.matrix for h in H], np.int32), _i)
        d.h_surface = _p(arr([h.surface for h in H], np.float32), _f)
        d.h_grid = _p(arr([h.grid for h in H], np.int32), _i)
        offs, cs, ns = [], [], []
        for h in H:
            if h.local_centers:
                offs.append(len(cs))
                cs.extend(h.local_centers)
                ns.extend(h.local_normals)
            else:
                offs.append(-1)
        d.h_local_off = _p(arr(offs, np.int32), _i)
        d.local_centers = _p(arr(cs if cs else [[0, 0, 0]], np.float32), _f)
        d.local_normals = _p(arr(ns if ns else [[0, 0, 0]], np.float32), _f)
        self._desc = d
        self.precision = precision
        self.h = lib().oracle_create(ctypes.byref(d), precision)
        c = np.zeros(3, np.int32)
        lib().oracle_counts(self.h, _p(c, _i))
        self.num_receivers, self.num_grids, self.num_heliostats = map(int, c)
        self.pool_size = d.groups * d.per_group

    @classmethod
    def from_files(cls, scene_path, config_path, precision: int = 32):
        sc = scene_text.parse_scene(Path(scene_path).read_text())
        cfg, _ = scene_text.parse_config(Path(config_path).read_text())
        return cls(sc, cfg, precision)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().oracle_free(h)
            self.h = None

    def receiver(self, i):
        ints = np.zeros(3, np.int32)
        vals = np.zeros(19, np.float64)
        lib().oracle_receiver(self.h, i, _p(ints, _i), _p(vals, _d))
        return {"type": int(ints[0]), "width": int(ints[1]), "height": int(ints[2]), "pixel_length": vals[0],
                "vertices": vals[1:13].reshape(4, 3), "normal": vals[13:16], "focus": vals[16:19]}

    def heliostat(self, i):
        ints = np.zeros(5, np.int32)
        vals = np.zeros(5, np.float64)
        lib().oracle_heliostat(self.h, i, _p(ints, _i), _p(vals, _d))
        return {"type": int(ints[0]), "grid": int(ints[1]), "num_facets": int(ints[2]), "num_sub": int(ints[3]),
                "sub_begin": int(ints[4]), "normal": vals[0:3], "focus_length": vals[3], "factor": vals[4]}

    def grid(self, i):
        ints = np.zeros(5, np.int32)
        lib().oracle_grid(self.h, i, _p(ints, _i))
        cells = tuple(int(x) for x in ints[:3])
        nnz, nsub = int(ints[3]), int(ints[4])
        index = np.zeros(cells[0] * cells[1] * cells[2] + 1, np.int32)
        match = np.zeros(max(nnz, 1), np.int32)
        lib().oracle_grid_csr(self.h, i, _p(index, _i), _p(match, _i))
        verts = np.zeros((max(nsub, 1) * 3, 3), np.float64)
        lib().oracle_grid_vertices(self.h, i, _p(verts, _d))
        return {"cells": cells, "index": index, "match": match[:nnz], "vertices": verts[: nsub * 3]}

    def facets(self, i):
        n = self.heliostat(i)["num_facets"]
        o = np.zeros((max(n, 1), 3), np.float64)
        nn = np.zeros((max(n, 1), 3), np.float64)
        lib().oracle_facets(self.h, i, _p(o, _d), _p(nn, _d))
        return o[:n], nn[:n]

    def receiver_hit(self, recv, origin, direction):
        o = np.asarray(origin, np.float32)
        d = np.asarray(direction, np.float32)
        tuv = np.zeros(3, np.float32)
        hit = lib().oracle_receiver_hit(self.h, recv, _p(o, _f), _p(d, _f), _p(tuv, _f))
        return bool(hit), tuv

    def walk(self, grid, own_begin, own_n, origin, direction):
        o = np.asarray(origin, np.float64)
        d = np.asarray(direction, np.float64)
        return bool(lib().oracle_walk(self.h, grid, own_begin, own_n, _p(o, _d), _p(d, _d)))

    def trace(self, ids, pool_dirs, pool_pert, offsets, light_begin=0, light_end=None, facet_stride=1,
              facet_phase=0, images=True, record=None, threads=0, record_only=False):
        """Trace heliostats `ids`.  offsets: dict heliostat -> int array of
        num_facets + 1.  record = (heliostat, facet_begin, facet_end) returns
        per-ray codes; with record_only that heliostat traces only the
        recorded facets (images, powers and counters then cover just those).
        Returns dict(images=[per receiver 2D], power, counters, records)."""
        ids = np.ascontiguousarray(np.array(ids, np.int32))
        P = self.pool_size
        dirs = np.ascontiguousarray(np.asarray(pool_dirs, np.float32).reshape(P, 3))
        pert = np.ascontiguousarray(np.asarray(pool_pert, np.float32).reshape(P, 3))
        nf = [self.heliostat(i)["num_facets"] for i in range(self.num_heliostats)]
        base = np.zeros(self.num_heliostats, np.int64)
        chunks = []
        pos = 0
        for h in range(self.num_heliostats):
            base[h] = pos
            if h in offsets:
                o = np.asarray(offsets[h], np.int32)
                assert o.size == nf[h] + 1
            else:
                o = np.zeros(nf[h] + 1, np.int32)
            chunks.append(o)
            pos += o.size
        offs = np.ascontiguousarray(np.concatenate(chunks).astype(np.int32))
        recs = [self.receiver(r) for r in range(self.num_receivers)]
        img_base = np.zeros(self.num_receivers + 1, np.int64)
        for r, rc in enumerate(recs):
            img_base[r + 1] = img_base[r] + rc["width"] * rc["height"]
        img = np.zeros(max(int(img_base[-1]), 1), np.float64)
        power = np.zeros(self.num_heliostats, np.float64)
        counters = np.zeros(12, np.int64)
        le = self.config["num_per_sunshape_group"] if light_end is None else light_end
        a = TraceArgs()
        a.ids = _p(ids, _i)
        a.n_ids = ids.size
        a.pool_dirs = _p(dirs, _f)
        a.pool_pert = _p(pert, _f)
        a.pool_size = P
        a.offsets = _p(offs, _i)
        a.offset_base = _p(base, ctypes.c_longlong)
        a.light_begin = light_begin
        a.light_end = le
        a.facet_stride = facet_stride
        a.facet_phase = facet_phase
        a.images = _p(img, _d) if images else None
        a.image_base = _p(img_base, ctypes.c_longlong)
        a.power = _p(power, _d)
        a.counters = _p(counters, ctypes.c_longlong)
        rec = None
        if record is not None:
            rid, fb, fe = record
            rec = np.full((fe - fb) * (le - light_begin), -4, np.int32)
            a.rec_id, a.rec_facet_begin, a.rec_facet_end = rid, fb, fe
            a.records = _p(rec, _i)
        else:
            a.rec_id, a.rec_facet_begin, a.rec_facet_end = -1, 0, 0
            a.records = None
        a.threads = threads
        a.record_only = 1 if (record is not None and record_only) else 0
        lib().oracle_trace(self.h, ctypes.byref(a))
        images_out = []
        for r, rc in enumerate(recs):
            images_out.append(img[img_base[r]:img_base[r + 1]].reshape(rc["height"], rc["width"]).copy())
        names = ["rays", "shadowed", "blocked", "missed", "hit", "clamped", "capped", "cells",
                 "tests_det", "tests_u", "tests_v", "tests_t"]
        return {"images": images_out, "power": power, "counters": dict(zip(names, map(int, counters))),
                "records": rec}


def smooth(image: np.ndarray, radius: int, ratio: float) -> np.ndarray:
    img = np.ascontiguousarray(image, np.float32)
    out = np.zeros_like(img)
    h, w = img.shape
    lib().oracle_smooth(_p(img, _f), _p(out, _f), w, h, radius, ratio)
    return out


def buie_theta(csr: float, groups: int, uniforms: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(uniforms, np.float32)
    out = np.zeros_like(u)
    lib().oracle_buie(csr, groups, _p(u, _f), _p(out, _f), u.size)
    return out


def buie_table(csr: float, groups: int):
    cx = np.zeros(groups + 1, np.float32)
    cy = np.zeros(groups + 1, np.float32)
    k = np.zeros(groups, np.float32)
    sc = np.zeros(5, np.float32)
    lib().oracle_buie_table(csr, groups, _p(cx, _f), _p(cy, _f), _p(k, _f), _p(sc, _f))
    return {"cdf_x": cx, "cdf_y": cy, "k": k, "less_465": sc[0], "gamma": sc[1], "A": sc[2], "B": sc[3], "C": sc[4]}


def sobol2(seed: int, first: int, n: int) -> np.ndarray:
    out = np.zeros((n, 2), np.uint32)
    lib().oracle_sobol2(seed & 0xFFFFFFFF, first, n, _p(out, ctypes.c_uint32))
    return out


def facet_offsets(seed: int, heliostat: int, n: int, pool: int) -> np.ndarray:
    out = np.zeros(n, np.int32)
    lib().oracle_facet_offsets(seed & 0xFFFFFFFF, heliostat, n, pool, _p(out, _i))
    return out


def mix32(x: int) -> int:
    return int(lib().oracle_mix32(x & 0xFFFFFFFF))


def default_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


# ---- single-routine probes (known-answer checks) ---------------------------
def probe_heliostat(type_, size, gap, matrix, px, normal, pos, focus_length=-1.0, cap=1 << 16):
    L = lib()
    f3 = lambda v: np.ascontiguousarray(v, np.float32)  # noqa: E731
    size, gap, normal, pos = f3(size), f3(gap), f3(normal), f3(pos)
    matrix = np.ascontiguousarray(matrix, np.int32)
    o = np.zeros((cap, 3), np.float32)
    n = np.zeros((cap, 3), np.float32)
    nsub = int(matrix[0] * matrix[1]) if type_ == 1 else 1
    sv = np.zeros((3 * nsub, 3), np.float32)
    lc = np.zeros((max(nsub, 1), 3), np.float32)
    ln = np.zeros((max(nsub, 1), 3), np.float32)
    counts = np.zeros(2, np.int32)
    L.oracle_probe_heliostat.argtypes = [_i, _pf, _pf, _pi, _f, _pf, _pf, _f, _i, _pf, _pf, _pf, _pf, _pf, _pi]
    rc = L.oracle_probe_heliostat(type_, _p(size, _f), _p(gap, _f), _p(matrix, _i), px, _p(normal, _f), _p(pos, _f),
                                  focus_length, cap, _p(o, _f), _p(n, _f), _p(sv, _f), _p(lc, _f), _p(ln, _f),
                                  _p(counts, _i))
    if rc != 0:
        raise ValueError("too many facets")
    nf = int(counts[0])
    return {"origins": o[:nf], "normals": n[:nf], "subverts": sv, "local_centers": lc, "local_normals": ln}


def probe_cylinder_hit(pos, size, origin, direction):
    L = lib()
    L.oracle_probe_cylinder_hit.argtypes = [_pf, _pf, _pf, _pf, _pf]
    a = [np.ascontiguousarray(v, np.float32) for v in (pos, size, origin, direction)]
    tuv = np.zeros(3, np.float32)
    hit = L.oracle_probe_cylinder_hit(*[_p(x, _f) for x in a], _p(tuv, _f))
    return bool(hit), tuv


def probe_cylinder_focus(pos, size, helio):
    L = lib()
    L.oracle_probe_cylinder_focus.argtypes = [_pf, _pf, _pf, _pf]
    a = [np.ascontiguousarray(v, np.float32) for v in (pos, size, helio)]
    out = np.zeros(3, np.float32)
    L.oracle_probe_cylinder_focus(*[_p(x, _f) for x in a], _p(out, _f))
    return out


def probe_cylinder_resolution(size, ppm):
    L = lib()
    L.oracle_probe_cylinder_resolution.argtypes = [_pf, _i, _pi]
    s = np.ascontiguousarray(size, np.float32)
    out = np.zeros(2, np.int32)
    L.oracle_probe_cylinder_resolution(_p(s, _f), ppm, _p(out, _i))
    return tuple(int(x) for x in out)


def probe_grid(pos, size, inter, helio_pos, helio_size, nsub, cap=1 << 16):
    L = lib()
    L.oracle_probe_grid.argtypes = [_pf, _pf, _pf, _i, _pf, _pf, _pi, _i, _pi, _pi, _pi]
    p3 = [np.ascontiguousarray(v, np.float32) for v in (pos, size, inter)]
    hp = np.ascontiguousarray(helio_pos, np.float32)
    hs = np.ascontiguousarray(helio_size, np.float32)
    ns = np.ascontiguousarray(nsub, np.int32)
    index = np.zeros(cap, np.int32)
    match = np.zeros(cap, np.int32)
    counts = np.zeros(4, np.int32)
    rc = L.oracle_probe_grid(*[_p(x, _f) for x in p3], len(ns), _p(hp, _f), _p(hs, _f), _p(ns, _i), cap,
                             _p(index, _i), _p(match, _i), _p(counts, _i))
    if rc != 0:
        raise ValueError("grid too large")
    ncell = int(counts[0] * counts[1] * counts[2])
    return index[: ncell + 1], match[: counts[3]]
