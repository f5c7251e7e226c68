"""ctypes binding of libqmcrt.so (include/qmcrt.h).

The shared library is built in-tree by solarenergy_chier_b200/build.py.  There
is no fallback: if the library is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libqmcrt.so"

QMCRT_OK = 0
ERRORS = {1: "invalid argument", 2: "I/O or format error", 3: "CUDA error", 4: "state error", 5: "out of memory"}

_i = ctypes.c_int
_u = ctypes.c_uint
_f = ctypes.c_float
_vp = ctypes.c_void_p
_pi = ctypes.POINTER(ctypes.c_int)
_pf = ctypes.POINTER(ctypes.c_float)
_pd = ctypes.POINTER(ctypes.c_double)
_pull = ctypes.POINTER(ctypes.c_ulonglong)


class SceneInfo(ctypes.Structure):
    _fields_ = [
        ("num_receivers", _i), ("num_grids", _i), ("num_heliostats", _i),
        ("num_sunshape_groups", _i), ("num_per_sunshape_group", _i), ("pool_size", _i),
        ("inverse_transform_sampling_groups", _i), ("config_fields", _i),
        ("sun_dir", _f * 3), ("dni", _f), ("csr", _f), ("receiver_pixel_length", _f),
        ("helio_disturb_std", _f), ("helio_pixel_length", _f), ("helio_reflected_rate", _f),
        ("ground_length", _f), ("ground_width", _f), ("total_facets", ctypes.c_longlong),
    ]


class QmcrtError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what} ({ERRORS.get(code, code)})")
        self.code = code


# name -> (restype, argtypes)
PROTOTYPES = {
    "qmcrt_last_error": (ctypes.c_char_p, []),
    "qmcrt_version": (_i, []),
    "qmcrt_debug_fail_allocations": (_i, [ctypes.c_longlong]),
    "qmcrt_scene_load": (_i, [ctypes.c_char_p, ctypes.c_char_p, _i, _u, ctypes.POINTER(_vp)]),
    "qmcrt_scene_free": (None, [_vp]),
    "qmcrt_scene_set_sun": (_i, [_vp, _pf]),
    "qmcrt_scene_get_info": (_i, [_vp, ctypes.POINTER(SceneInfo)]),
    "qmcrt_receiver_get": (_i, [_vp, _i, _pi, _pi, _pi, _pf, _pf, _pf, _pf]),
    "qmcrt_heliostat_get": (_i, [_vp, _i, _pi, _pi, _pi, _pi, _pi, _pf, _pf, _pf, _pf]),
    "qmcrt_grid_get": (_i, [_vp, _i, _pi, _pi, _pi, _pi, _pi, _pi]),
    "qmcrt_grid_csr": (_i, [_vp, _i, _pi, _pi]),
    "qmcrt_grid_vertices": (_i, [_vp, _i, _pf]),
    "qmcrt_heliostat_facets": (_i, [_vp, _i, _pf, _pf]),
    "qmcrt_set_sample_pool": (_i, [_vp, _vp, _vp, _i, _i, _i]),
    "qmcrt_generate_sample_pool": (_i, [_vp, _u, _i, _f]),
    "qmcrt_get_sample_pool": (_i, [_vp, _pf, _pf]),
    "qmcrt_set_facet_offsets": (_i, [_vp, _i, _pi, _i]),
    "qmcrt_get_facet_offsets": (_i, [_vp, _i, _pi, _i]),
    "qmcrt_generate_facet_offsets": (_i, [_vp, _u]),
    "qmcrt_set_math_mode": (_i, [_vp, _i]),
    "qmcrt_set_light_range": (_i, [_vp, _i, _i]),
    "qmcrt_trace_heliostat": (_i, [_vp, _i, _vp]),
    "qmcrt_trace_heliostats": (_i, [_vp, _pi, _i, _vp]),
    "qmcrt_receiver_image": (_i, [_vp, _i, _pf, _pi, _pi]),
    "qmcrt_receiver_device_image": (_i, [_vp, _i, ctypes.POINTER(_vp), _pi, _pi]),
    "qmcrt_receiver_clear": (_i, [_vp, _i, _vp]),
    "qmcrt_power_fp64": (_i, [_vp, _pd, _pd]),
    "qmcrt_power_clear": (_i, [_vp]),
    "qmcrt_diagnostics": (_i, [_vp, _pull]),
    "qmcrt_debug_hit_records": (_i, [_vp, _i, _i, _i, _i, _i, _pi]),
    "qmcrt_debug_hit_bits": (_i, [_vp, _pi, _i, _vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong), _vp]),
    "qmcrt_debug_shadow_free": (_i, [_vp, _pi]),
    "qmcrt_debug_block_free": (_i, [_vp, _i, _pi]),
    "qmcrt_smooth": (_i, [_vp, _i, _i, _i, _f, _vp]),
    "qmcrt_smooth_static": (_i, [_vp, _i, _i, _i, _f, _vp]),
    "qmcrt_load_tasks": (_i, [_vp, ctypes.c_char_p, _pi, _pi, _i, _pi, _pi, _pi]),
    "qmcrt_save_text": (_i, [ctypes.c_char_p, _i, _i, _pf, _i, _pf]),
    "qmcrt_pipeline_run": (_i, [_i, ctypes.POINTER(ctypes.c_char_p)]),
    "qmcrt_batch_create": (_i, [ctypes.POINTER(_vp), _i, _pi, _pf, _i, ctypes.POINTER(_vp)]),
    "qmcrt_batch_free": (None, [_vp]),
    "qmcrt_batch_set_suns": (_i, [_vp, _pf, _vp]),
    "qmcrt_batch_set_light_range": (_i, [_vp, _i, _i]),
    "qmcrt_batch_set_math_mode": (_i, [_vp, _i]),
    "qmcrt_batch_info": (_i, [_vp, _pi, _pi, ctypes.POINTER(ctypes.c_longlong)]),
    "qmcrt_batch_trace": (_i, [_vp, _vp]),
    "qmcrt_batch_capture_graph": (_i, [_vp, _i]),
    "qmcrt_batch_graph_launch": (_i, [_vp, _vp]),
    "qmcrt_batch_clear": (_i, [_vp, _vp]),
    "qmcrt_batch_image": (_i, [_vp, _i, _i, _pf, _pi, _pi]),
    "qmcrt_batch_power_fp64": (_i, [_vp, _i, _pd, _pd]),
    "qmcrt_batch_autotune": (_i, [_vp, _vp, _pi, _pf]),
    "qmcrt_batch_autotune_shapes": (_i, [_vp, _vp, _pi, _pf]),
    "qmcrt_batch_set_launch_shape": (_i, [_vp, _i]),
    "qmcrt_launch_shapes": (_i, [_pi, _pi, _pi, _pi]),
    "qmcrt_set_launch_shape": (_i, [_vp, _i]),
    "qmcrt_autotune": (_i, [_vp, _pi, _i, _vp, _pi, _pf]),
    "qmcrt_batch_debug_geometry": (_i, [_vp, _i, _i, _pf, _pf]),
    "qmcrt_diff_create": (_i, [_vp, _f, ctypes.POINTER(_vp)]),
    "qmcrt_diff_free": (None, [_vp]),
    "qmcrt_diff_set_params": (_i, [_vp, _pf, _pf]),
    "qmcrt_diff_set_target": (_i, [_vp, _i, _pf]),
    "qmcrt_diff_set_light_range": (_i, [_vp, _i, _i]),
    "qmcrt_fwd": (_i, [_vp, _pd, _vp]),
    "qmcrt_bwd": (_i, [_vp, _pd, _vp]),
    "qmcrt_diff_flux": (_i, [_vp, _i, _pf, _pi, _pi]),
    "qmcrt_diff_plain": (_i, [_vp, _vp]),
    "qmcrt_diff_image": (_i, [_vp, _i, _pf, _pi, _pi]),
    "qmcrt_diff_power": (_i, [_vp, _pd, _pd]),
    "qmcrt_config_check": (_i, [ctypes.c_char_p, _pi]),
    "qmcrt_grid_build_device": (_i, [_vp, _i, _pf]),
    "qmcrt_debug_grid_cells": (_i, [_vp, _i, _pi, _pi, ctypes.POINTER(ctypes.c_longlong)]),
    "qmcrt_diff_create_suns": (_i, [_vp, _pf, _i, _f, ctypes.POINTER(_vp)]),
    "qmcrt_diff_set_hit_records": (_i, [_vp, _i, ctypes.c_longlong]),
    "qmcrt_diff_hit_records": (_i, [_vp, _pi, ctypes.POINTER(ctypes.c_longlong)]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load libqmcrt.so (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: run `python -m solarenergy_chier_b200.build` "
                          "(or __graft_entry__.build()) first")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code: int) -> None:
    if code != QMCRT_OK:
        msg = load().qmcrt_last_error().decode(errors="replace")
        raise QmcrtError(code, msg)
