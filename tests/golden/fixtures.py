"""Deterministic inputs shared by make_golden.py and the tests that replay
its fixtures: per-facet pool offsets from a splitmix64 hash (integer
arithmetic only, so identical on every machine)."""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def hash_offsets(n: int, pool_size: int, seed: int) -> np.ndarray:
    """n offsets in [0, pool_size) from splitmix64(seed * golden + index)."""
    with np.errstate(over="ignore"):
        x = np.arange(n, dtype=np.uint64) + np.uint64(seed) * _GOLDEN
        x = x + _GOLDEN
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
        hi = x >> np.uint64(32)
        return ((hi * np.uint64(pool_size)) >> np.uint64(32)).astype(np.int32)


def offsets_for(num_facets: list[int], pool_size: int, seed: int) -> dict:
    return {h: hash_offsets(n + 1, pool_size, seed * 1000003 + h) for h, n in enumerate(num_facets)}
