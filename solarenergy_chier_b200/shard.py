"""One trace split over several GPUs: one process per GPU, rays sharded, flux maps added.

The reference traces a field one heliostat at a time on one GPU
(RayTracingPipeline.cpp:66-81 calling QuasiMonteCarloRayTracer::rayTracing,
QuasiMonteCarloRayTracer.cpp:15-91).  Rays are independent and their energy
only adds into the receiver images and the per-heliostat powers, so a field
shards without any exchange during tracing:

* by heliostat ("heliostats"): each rank traces a subset of the heliostats,
  balanced by micro-facet count (every facet carries the same number of rays);
* by light index ("lights"): each rank traces every heliostat for a
  contiguous range of the light indexes l of the reference's (facet, light)
  grid (RectangleReceiverRectangleGridRayTracing.cu:6-41).

After tracing, one sum-reduce of each float32 receiver image to the
destination rank and one FP64 sum all-reduce of the per-heliostat powers
(the total is recomputed from them) give every number a single-GPU trace
gives, up to the order of the float additions.  All ranks must hold the same scene, sample pool and facet
offsets (load with the same seed, or inject the same pools).

The collectives go through ``torch.distributed`` (NCCL over NVLink on the
GPUs, gloo on the host); the functions here take whatever tensors they are
given, so the host-side logic is the same for both.
"""
from __future__ import annotations

import heapq
from typing import Sequence

import numpy as np

SPLITS = ("heliostats", "lights")


def heliostat_shards(facet_counts: Sequence[int], world: int) -> list[list[int]]:
    """Heliostat ids of every rank, balanced by facet count.

    Largest first onto the least loaded rank (ties: lowest rank, then lowest
    heliostat id), so every rank computes the same assignment.  Each rank's
    ids come back in increasing order.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    counts = [int(c) for c in facet_counts]
    if any(c < 0 for c in counts):
        raise ValueError("facet counts must be >= 0")
    order = sorted(range(len(counts)), key=lambda h: (-counts[h], h))
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for h in order:
        load, r = heapq.heappop(heap)
        out[r].append(h)
        heapq.heappush(heap, (load + counts[h], r))
    return [sorted(ids) for ids in out]


def light_shards(lights: int, world: int) -> list[tuple[int, int]]:
    """[begin, end) light-index range of every rank: contiguous, sizes differing by at most one."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if lights < 0:
        raise ValueError("lights must be >= 0")
    q, r = divmod(lights, world)
    out, b = [], 0
    for k in range(world):
        e = b + q + (1 if k < r else 0)
        out.append((b, e))
        b = e
    return out


def compensated_sum(values) -> float:
    """Neumaier-compensated sum, in the order given (the total that
    qmcrt_power_fp64 reports for the same per-heliostat powers)."""
    total, comp = 0.0, 0.0
    for x in values:
        x = float(x)
        t = total + x
        comp += (total - t) + x if abs(total) >= abs(x) else (x - t) + total
        total = t
    return total + comp


def reduce_flux(images, per_heliostat, group=None, dst: int = 0):
    """Add every rank's partial flux maps and powers.

    images: tensors, summed in place onto rank ``dst`` (other ranks' copies
    are left partial); per_heliostat: tensor of this rank's per-heliostat
    powers.  Returns (images, per-heliostat FP64 powers summed on every rank,
    their compensated total).  With a heliostat split every heliostat's power
    comes from one rank and the others add zeros, so powers and total equal a
    single-GPU trace's bit for bit.
    """
    import torch
    import torch.distributed as dist

    per = per_heliostat.to(torch.float64).reshape(-1).clone()
    if dist.is_initialized():
        for img in images:
            dist.reduce(img, dst, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(per, op=dist.ReduceOp.SUM, group=group)
    return images, per, compensated_sum(per.cpu().numpy())


def device_image_tensor(scene, receiver: int = 0):
    """A torch view (no copy) of a receiver's float32 device image, rows = height.

    The view does not own the memory: it is valid while the scene lives.
    """
    import torch

    ptr, w, h = scene.device_image(receiver)

    class _View:
        __cuda_array_interface__ = {"shape": (h, w), "typestr": "<f4", "data": (ptr, False), "version": 3,
                                    "strides": None}

    return torch.as_tensor(_View(), device=f"cuda:{torch.cuda.current_device()}")


class ShardedTrace:
    """This rank's part of a field trace split over a process group.

    ``trace`` traces the rank's share on its own GPU (no collective);
    ``reduce`` then adds the shares: receiver images on rank ``dst``, powers
    on every rank.
    """

    def __init__(self, scene, split: str = "heliostats", group=None):
        import torch.distributed as dist

        if split not in SPLITS:
            raise ValueError(f"split must be one of {SPLITS}")
        self.scene = scene
        self.split = split
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1

    def share(self, heliostats: Sequence[int]) -> tuple[list[int], tuple[int, int]]:
        """(heliostat ids, light range) this rank traces for a trace of ``heliostats``."""
        ids = [int(h) for h in heliostats]
        L = self.scene.lights_per_group
        if self.split == "heliostats":
            counts = [self.scene.heliostat(h)["num_facets"] for h in ids]
            mine = heliostat_shards(counts, self.world)[self.rank]
            return [ids[k] for k in mine], (0, L)
        return ids, light_shards(L, self.world)[self.rank]

    def trace(self, heliostats: Sequence[int], stream=None) -> None:
        ids, (lb, le) = self.share(heliostats)
        self.scene.set_light_range(lb, le)
        if ids and le > lb:
            self.scene.trace(ids, stream)

    def reduce(self, dst: int = 0, stream=None):
        """Sum the shares.  Returns (images as tensors, complete on ``dst``;
        per-heliostat FP64 powers; total power)."""
        import torch

        per, _ = self.scene.power()
        if stream is not None:
            torch.cuda.current_stream().wait_stream(stream)
        images = [device_image_tensor(self.scene, r) for r in range(self.scene.num_receivers)]
        per_t = torch.from_numpy(np.ascontiguousarray(per)).to(images[0].device if images else "cuda")
        return reduce_flux(images, per_t, group=self.group, dst=dst)
