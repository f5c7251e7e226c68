"""Roofline denominators measured on the running GPU (include/qmcrt_bench.h)."""
from __future__ import annotations

import ctypes

from ._lib import check, load


def fp32_fma_tflops() -> float:
    lib = load()
    fn = lib.qmcrt_microbench_fp32
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(ctypes.c_double)]
    out = ctypes.c_double()
    check(fn(ctypes.byref(out)))
    return out.value


def l2_atomics_per_s(n_pixels: int) -> float:
    lib = load()
    fn = lib.qmcrt_microbench_atomics
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    out = ctypes.c_double()
    check(fn(int(n_pixels), ctypes.byref(out)))
    return out.value * 1e9
