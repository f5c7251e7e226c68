"""CPU stand-ins for the per-rank objects of the sharded batch and adjoint
tests (tests/test_shard.py): the same interfaces as the product's Batch and
Diff, computed on the host, so the split and reduction logic of
solarenergy_chier_b200.shard runs as gloo ranks without a GPU."""
import json
from pathlib import Path

import numpy as np

from oracle import oracle
from tests.shard_inputs import inputs

LIGHTS = 4


class OracleBatch:
    """Instances (scene index, sun) traced by the CPU oracle; each instance
    loads its scene with the configuration's sun replaced by its own."""

    def __init__(self, scenes, instances, workdir):
        self.items = []
        for k, (si, sun) in enumerate(instances):
            scene_path, config_path = scenes[si]
            cfg = json.loads(Path(config_path).read_text())
            cfg["sun_dir"] = [float(x) for x in sun]
            path = Path(workdir) / f"sun_{si}_{'_'.join(f'{x:.6f}' for x in sun)}.json"
            path.write_text(json.dumps(cfg))
            self.items.append(oracle.OracleScene.from_files(scene_path, path))
        self.results = [None] * len(self.items)

    def trace(self, stream=None):
        for k, o in enumerate(self.items):
            dirs, pert, offsets = inputs(o)
            self.results[k] = o.trace(list(range(o.num_heliostats)), dirs, pert, offsets, 0, LIGHTS, threads=2)

    def image(self, k, r):
        return self.results[k]["images"][r]

    def power(self, k):
        p = self.results[k]["power"]
        return p, float(p.sum())


class LinearPair:
    """A differentiable pair whose flux at sun k is a fixed seeded linear map
    of the H x 4 parameters (one receiver of `pixels` values per sun): loss =
    sum over suns of |A_k theta - target_k|^2, gradient 2 A_k^T (A_k theta -
    target_k); parameters shared by the suns, as in the product's pair."""

    def __init__(self, suns, heliostats, pixels=40):
        self.suns = np.asarray(suns, np.float64).reshape(-1, 3)
        self.H = heliostats
        self.A = []
        for s in self.suns:
            rng = np.random.default_rng(int(abs(s).sum() * 1e6) % (2 ** 32))
            self.A.append(rng.standard_normal((pixels, heliostats * 4)))
        self.targets = [np.zeros(pixels) for _ in self.suns]
        self.theta = np.zeros(heliostats * 4)

    def set_params(self, aim=None, normal=None):
        t = np.zeros((self.H, 4))
        if aim is not None:
            t[:, :2] = np.asarray(aim, np.float64).reshape(self.H, 2)
        if normal is not None:
            t[:, 2:] = np.asarray(normal, np.float64).reshape(self.H, 2)
        self.theta = t.ravel()

    def set_target(self, target, receiver=0):
        self.targets[receiver] = np.asarray(target, np.float64).ravel()

    def set_light_range(self, begin, end):
        pass

    def forward(self, stream=None):
        return float(sum(((A @ self.theta - t) ** 2).sum() for A, t in zip(self.A, self.targets)))

    def backward(self, stream=None):
        g = sum(2 * A.T @ (A @ self.theta - t) for A, t in zip(self.A, self.targets))
        return np.asarray(g).reshape(self.H, 4)
