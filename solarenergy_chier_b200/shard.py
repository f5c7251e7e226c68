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

Batched tracing shards whole (scene, sun) instances (ShardedBatch: balanced
by rays, no exchange while tracing, one gather of each instance's images and
powers at the end).  The differentiable pair over several suns shards the
suns (ShardedDiff): the loss sums over suns and the parameters are shared,
so one all-reduce of the loss and one FP64 all-reduce of the heliostats x 4
gradient give every rank the one-pair result.

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


# ---- batched tracing: (scene, sun) instances split over ranks -------------------
def instance_shards(rays_per_instance: Sequence[int], world: int) -> list[list[int]]:
    """Instance indexes of every rank, balanced by rays (largest first onto the
    least loaded rank, as heliostat_shards)."""
    return heliostat_shards(rays_per_instance, world)


def gather_instances(results: dict, group=None, dst: int = 0):
    """Collect every rank's per-instance results on rank ``dst``.

    results: {instance index: (images, per-heliostat FP64 powers, total)} of
    this rank's instances.  Returns, on ``dst``, the union over the ranks
    (None elsewhere).  Instances belong to one rank each, so nothing is added:
    every number is the one its rank computed."""
    import torch.distributed as dist

    if not dist.is_initialized():
        return dict(results)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    out = [None] * world if rank == dst else None
    dist.gather_object(dict(results), out, dst=dst, group=group)
    if rank != dst:
        return None
    merged = {}
    for part in out:
        overlap = set(merged) & set(part)
        if overlap:
            raise RuntimeError(f"instances traced by two ranks: {sorted(overlap)}")
        merged.update(part)
    return merged


class ShardedBatch:
    """A batch of (scene, sun) instances split over a process group.

    Every rank builds a batch of its own share of the instances (balanced by
    rays: instance_shards) and traces it with no collective; ``gather`` then
    brings each instance's receiver images and FP64 powers to rank ``dst``
    (one gather, no reduction: an instance is traced by exactly one rank).
    ``make_batch(scenes, instances)`` builds the rank's batch (default: the
    product's Batch)."""

    def __init__(self, scenes, instances, rays_per_instance: Sequence[int], group=None, make_batch=None):
        import torch.distributed as dist

        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.group = group
        if len(rays_per_instance) != len(instances):
            raise ValueError("one ray count per instance")
        self.mine = instance_shards(rays_per_instance, self.world)[self.rank]
        if make_batch is None:
            from .scene import Batch as make_batch
        self.batch = make_batch(scenes, [instances[k] for k in self.mine]) if self.mine else None

    def trace(self, stream=None) -> None:
        if self.batch is not None:
            self.batch.trace(stream)

    def gather(self, num_receivers, dst: int = 0):
        results = {}
        for local, k in enumerate(self.mine):
            images = [self.batch.image(local, r) for r in range(num_receivers(k))]
            per, total = self.batch.power(local)
            results[k] = (images, per, total)
        return gather_instances(results, self.group, dst)


# ---- differentiation: suns split over ranks ---------------------------------------
def sun_shards(num_suns: int, world: int) -> list[tuple[int, int]]:
    """[begin, end) sun range of every rank (contiguous, sizes within one)."""
    return light_shards(num_suns, world)


class ShardedDiff:
    """The differentiable pair over several suns, split over a process group.

    The loss sums over the suns and the parameters (aim and normal offsets
    per heliostat) are shared, so each rank builds the pair over its own
    contiguous share of the suns (sun_shards); ``forward`` adds the ranks'
    losses (one FP64 all-reduce of a scalar) and ``backward`` their
    gradients (one FP64 all-reduce over the heliostats x 4 parameters).
    Every rank ends with the loss and gradient one pair over all suns gives,
    up to the order of the additions.  ``make_pair(suns)`` builds the rank's
    pair (default: the product's Diff over `scene`)."""

    def __init__(self, scene, suns, sigma_px: float = 2.0, group=None, make_pair=None):
        import torch.distributed as dist

        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.group = group
        suns = np.asarray(suns, np.float32).reshape(-1, 3)
        self.num_suns = suns.shape[0]
        self.begin, self.end = sun_shards(self.num_suns, self.world)[self.rank]
        if make_pair is None:
            from .scene import Diff

            def make_pair(s):
                return Diff(scene, sigma_px, suns=s)
        self.pair = make_pair(suns[self.begin:self.end]) if self.end > self.begin else None
        self.num_heliostats = scene.num_heliostats
        self.num_receivers = scene.num_receivers

    def owns(self, sun: int) -> bool:
        return self.begin <= sun < self.end

    def set_params(self, aim=None, normal=None) -> None:
        if self.pair is not None:
            self.pair.set_params(aim, normal)

    def set_target(self, target, sun: int, receiver: int = 0) -> None:
        """Target of receiver `receiver` at sun `sun` (kept by the rank that owns the sun)."""
        if not 0 <= sun < self.num_suns:
            raise ValueError("sun index out of range")
        if self.owns(sun):
            self.pair.set_target(target, receiver=(sun - self.begin) * self.num_receivers + receiver)

    def set_light_range(self, begin: int, end: int) -> None:
        if self.pair is not None:
            self.pair.set_light_range(begin, end)

    def _sum(self, values: np.ndarray) -> np.ndarray:
        import torch
        import torch.distributed as dist

        t = torch.from_numpy(np.ascontiguousarray(values, np.float64).copy())
        if dist.is_initialized():
            if dist.get_backend(self.group) == "nccl":
                t = t.cuda()
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy()

    def forward(self, stream=None) -> float:
        loss = self.pair.forward(stream) if self.pair is not None else 0.0
        return float(self._sum(np.array([loss]))[0])

    def backward(self, stream=None) -> np.ndarray:
        g = self.pair.backward(stream) if self.pair is not None else np.zeros((self.num_heliostats, 4))
        return self._sum(g)
