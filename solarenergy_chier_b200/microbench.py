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


def l2_atomics_replay_per_s(device_codes_ptr: int, n_codes: int, n_hits: int, n_pixels: int, repeats: int) -> float:
    """Float atomics per second when the tracer's recorded deposits (device
    array of n_codes outcome codes, n_hits of them pixels) are replayed."""
    lib = load()
    fn = lib.qmcrt_microbench_atomics_replay
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    ms = ctypes.c_double()
    check(fn(ctypes.c_void_p(device_codes_ptr), int(n_codes), int(n_pixels), int(repeats), ctypes.byref(ms)))
    return n_hits * repeats / (ms.value * 1e-3)


def primitive_mismatches(count: int = 1) -> list[int]:
    """Inputs (of all 2^32 float bit patterns) where the tracer's own
    correctly rounded primitives differ from CUDA's: [rsqrt, rsqrt without
    its range test on [2^-125, 2^125), division by a receiver height with its
    precomputed reciprocal, the cylinder's u from it, the square root from the
    reciprocal root, the Newton reciprocal, Markstein's division with it]."""
    lib = load()
    fn = lib.qmcrt_debug_check_primitives
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]
    out = (ctypes.c_ulonglong * count)()
    check(fn(out, count))
    return [int(v) for v in out]
