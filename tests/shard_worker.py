"""One gloo rank of the sharded-trace test (tests/test_shard.py).

Each rank traces its share of a small field with the CPU oracle, then
solarenergy_chier_b200.shard.reduce_flux adds the shares exactly as the GPU
path does after its kernels; rank 0 saves what it received.
argv: scene config split lights out.npz (RANK / WORLD_SIZE / MASTER_* from the env).
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


def main():
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
