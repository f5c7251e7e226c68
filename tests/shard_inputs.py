"""Seeded sample pool and facet offsets shared by the sharded-trace test and its gloo ranks."""
import numpy as np

from oracle import oracle


def inputs(o, seed: int = 5):
    """(pool directions, pool perturbations, offsets per heliostat) for OracleScene ``o``."""
    P = o.pool_size
    rng = np.random.default_rng(seed)
    th = 0.00465 * np.sqrt(rng.random(P))
    ph = 2 * np.pi * rng.random(P)
    dirs = np.stack([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)], 1).astype(np.float32)
    p = np.stack([rng.standard_normal(P) * 0.002, np.ones(P), rng.standard_normal(P) * 0.002], 1)
    pert = (p / np.linalg.norm(p, axis=1, keepdims=True)).astype(np.float32)
    offsets = {h: oracle.facet_offsets(seed, h, o.heliostat(h)["num_facets"] + 1, P) for h in range(o.num_heliostats)}
    return dirs, pert, offsets
