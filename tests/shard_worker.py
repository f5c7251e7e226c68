"""One gloo rank of the sharded-trace test (tests/test_shard.py).

Each rank traces its share of a small field with the CPU oracle, then
solarenergy_chier_b200.shard.reduce_flux adds the shares exactly as the GPU
path does after its kernels; rank 0 saves what it received.
argv: scene config split lights out.npz, or batch scene config out.npz, or diff
out.npz (RANK / WORLD_SIZE / MASTER_* from the env).
"""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import datetime  # noqa: E402

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from oracle import oracle  # noqa: E402
from solarenergy_chier_b200 import shard  # noqa: E402
from tests.shard_inputs import inputs  # noqa: E402


def batch_main(scene_path, config_path, out):
    """Instances (this field at several suns) split over the ranks by
    ShardedBatch, traced by the CPU oracle, gathered on rank 0."""
    from tests.shard_models import OracleBatch
    from solarenergy_chier_b200 import synth

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rank = dist.get_rank()
    suns = synth.sun_positions(days=2, hours=3)
    instances = [(0, s) for s in suns]
    rays = [1000 + 17 * k for k in range(len(instances))]
    workdir = Path(out).parent / f"rank{rank}"
    workdir.mkdir(exist_ok=True)
    sb = shard.ShardedBatch([(scene_path, config_path)], instances, rays,
                            make_batch=lambda sc, inst: OracleBatch(sc, inst, workdir))
    sb.trace()
    got = sb.gather(lambda k: 1)
    if rank == 0:
        np.savez(out, n=len(got), **{f"image{k}": v[0][0] for k, v in got.items()},
                 **{f"per{k}": v[1] for k, v in got.items()}, **{f"total{k}": v[2] for k, v in got.items()},
                 mine=np.array(sb.mine))
    dist.barrier()
    dist.destroy_process_group()


def diff_main(out):
    """Suns split over the ranks by ShardedDiff around the linear stand-in pair."""
    from tests.shard_models import LinearPair

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rank = dist.get_rank()
    H = 7
    suns = np.array([[0.1 * k, -1.0, 0.05 * k] for k in range(5)])

    class SceneStub:
        num_heliostats = H
        num_receivers = 1

    sd = shard.ShardedDiff(SceneStub(), suns, make_pair=lambda s: LinearPair(s, H))
    rng = np.random.default_rng(3)
    targets = [rng.standard_normal(40) for _ in range(len(suns))]
    for k, t in enumerate(targets):
        sd.set_target(t, sun=k)
    aim, nrm = rng.standard_normal((H, 2)), rng.standard_normal((H, 2))
    sd.set_params(aim, nrm)
    loss = sd.forward()
    grad = sd.backward()
    if rank == 0:
        np.savez(out, loss=loss, grad=grad, begin=sd.begin, end=sd.end)
    dist.barrier()
    dist.destroy_process_group()


def main():
    if sys.argv[1] == "batch":
        return batch_main(*sys.argv[2:5])
    if sys.argv[1] == "diff":
        return diff_main(sys.argv[2])
    scene_path, config_path, split, lights, out = sys.argv[1:6]
    lights = int(lights)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rank, world = dist.get_rank(), dist.get_world_size()
    o = oracle.OracleScene.from_files(scene_path, config_path)
    dirs, pert, offsets = inputs(o)
    ids = list(range(o.num_heliostats))
    if split == "heliostats":
        counts = [o.heliostat(h)["num_facets"] for h in ids]
        mine, (lb, le) = shard.heliostat_shards(counts, world)[rank], (0, lights)
    else:
        mine, (lb, le) = ids, shard.light_shards(lights, world)[rank]
    res = o.trace(mine, dirs, pert, offsets, light_begin=lb, light_end=le, threads=2) if mine and le > lb else None
    images = [torch.from_numpy(res["images"][r] if res else np.zeros((o.receiver(r)["height"], o.receiver(r)["width"])))
              for r in range(o.num_receivers)]
    per = torch.from_numpy(res["power"] if res else np.zeros(o.num_heliostats))
    images, per, total = shard.reduce_flux(images, per, dst=0)
    if rank == 0:
        np.savez(out, per=per.numpy(), total=total, mine=np.array(mine),
                 **{f"image{r}": im.numpy() for r, im in enumerate(images)})
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
