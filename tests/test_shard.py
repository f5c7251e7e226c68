"""Multi-GPU sharding of a trace (solarenergy_chier_b200/shard.py), on the host.

The shard assignment and the reduction that follow the GPU kernels are
exercised as two gloo ranks on the CPU: each rank traces its share of a small
field with the oracle and the shares are added by shard.reduce_flux.  Bar:
with a heliostat split, per-heliostat powers and the total equal a one-rank
trace bit for bit and images agree to FP64 summation order (1e-12); with a
light split, powers and images agree to 1e-12 relative.
"""
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from solarenergy_chier_b200 import shard, synth
from tests.shard_inputs import inputs

ROOT = Path(__file__).resolve().parents[1]
LIGHTS = 6


def test_heliostat_shards_cover_and_balance():
    rng = np.random.default_rng(0)
    counts = rng.integers(1000, 300_000, 624).tolist()
    for world in (1, 2, 3, 8):
        sh = shard.heliostat_shards(counts, world)
        assert len(sh) == world
        flat = sorted(h for ids in sh for h in ids)
        assert flat == list(range(624))
        assert all(ids == sorted(ids) for ids in sh)
        loads = [sum(counts[h] for h in ids) for ids in sh]
        # largest-first greedy: no rank exceeds the mean by more than one heliostat
        assert max(loads) - sum(loads) / world <= max(counts)
        assert sh == shard.heliostat_shards(counts, world)  # every rank computes the same split
    assert shard.heliostat_shards([5, 5], 4) == [[0], [1], [], []]
    assert shard.heliostat_shards([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard.heliostat_shards([1], 0)
    with pytest.raises(ValueError):
        shard.heliostat_shards([-1], 1)


def test_light_shards_partition_the_lights():
    for lights, world in ((2048, 1), (2048, 8), (2048, 3), (5, 8), (0, 2)):
        sh = shard.light_shards(lights, world)
        assert len(sh) == world and sh[0][0] == 0 and sh[-1][1] == lights
        assert all(a[1] == b[0] for a, b in zip(sh, sh[1:]))
        sizes = [e - b for b, e in sh]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.light_shards(4, 0)
    with pytest.raises(ValueError):
        shard.light_shards(-1, 2)


def test_compensated_sum_matches_fsum_on_cancelling_input():
    import math

    rng = np.random.default_rng(1)
    x = np.concatenate([rng.standard_normal(1000) * 1e12, rng.standard_normal(1000)])
    x = np.concatenate([x, -x[:1000]])
    assert shard.compensated_sum(x) == pytest.approx(math.fsum(x), abs=1e-6)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.fixture(scope="module")
def field(tmp_path_factory):
    d = tmp_path_factory.mktemp("shard")
    files = synth.small_field(d, seed=2, helio_pixel=0.1, rows=3, cols=4)
    o = oracle.OracleScene.from_files(files.scene, files.config)
    dirs, pert, offsets = inputs(o)
    full = o.trace(list(range(o.num_heliostats)), dirs, pert, offsets, light_begin=0, light_end=LIGHTS, threads=2)
    return files, o, full, d


def _run_ranks(files, split, out, world=2, argv=None):
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), WORLD_SIZE=str(world),
               OMP_NUM_THREADS="2")
    procs = []
    args = argv if argv is not None else [str(files.scene), str(files.config), split, str(LIGHTS), str(out)]
    for rank in range(world):
        e = dict(env, RANK=str(rank), LOCAL_RANK=str(rank))
        procs.append(subprocess.Popen([sys.executable, str(ROOT / "tests" / "shard_worker.py"), *args], env=e,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
    logs = []
    for p in procs:
        try:
            logs.append(p.communicate(timeout=180)[0].decode(errors="replace"))
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
    assert all(p.returncode == 0 for p in procs), "\n".join(logs)
    return np.load(out)


def test_heliostat_split_reduces_to_the_one_rank_trace(field):
    files, o, full, d = field
    r = _run_ranks(files, "heliostats", d / "h.npz")
    assert 0 < r["mine"].size < o.num_heliostats
    assert np.array_equal(r["per"], full["power"])
    assert float(r["total"]) == shard.compensated_sum(full["power"])
    for k in range(o.num_receivers):
        np.testing.assert_allclose(r[f"image{k}"], full["images"][k], rtol=1e-12, atol=1e-9)
    assert full["power"].sum() > 0


def test_light_split_reduces_to_the_one_rank_trace(field):
    files, o, full, d = field
    r = _run_ranks(files, "lights", d / "l.npz")
    np.testing.assert_allclose(r["per"], full["power"], rtol=1e-12)
    assert float(r["total"]) == pytest.approx(float(full["power"].sum()), rel=1e-12)
    for k in range(o.num_receivers):
        np.testing.assert_allclose(r[f"image{k}"], full["images"][k], rtol=1e-12, atol=1e-9)


def test_instance_shards_cover_and_balance():
    rays = [5, 9, 1, 7, 7, 3]
    sh = shard.instance_shards(rays, 2)
    assert sorted(k for ids in sh for k in ids) == list(range(6))
    loads = [sum(rays[k] for k in ids) for ids in sh]
    assert abs(loads[0] - loads[1]) <= max(rays)
    assert shard.sun_shards(32, 3) == [(0, 11), (11, 22), (22, 32)]


def test_batch_split_gathers_every_instance(field, tmp_path):
    """Instances (the field at 6 suns) split over two gloo ranks by
    ShardedBatch, each rank tracing its own with the CPU oracle: rank 0
    receives every instance, each equal to a one-rank trace of it."""
    from solarenergy_chier_b200 import synth as sy
    from tests.shard_models import OracleBatch

    files, o, full, d = field
    r = _run_ranks(files, None, tmp_path / "b.npz", argv=["batch", str(files.scene), str(files.config),
                                                           str(tmp_path / "b.npz")])
    suns = sy.sun_positions(days=2, hours=3)
    assert int(r["n"]) == len(suns)
    assert 0 < r["mine"].size < len(suns)
    one = OracleBatch([(files.scene, files.config)], [(0, s) for s in suns], tmp_path)
    one.trace()
    for k in range(len(suns)):
        assert np.array_equal(r[f"image{k}"], one.image(k, 0))
        assert np.array_equal(r[f"per{k}"], one.power(k)[0])


def test_sun_split_adjoint_reduces_to_one_pair(tmp_path):
    """The pair over 5 suns split over two gloo ranks by ShardedDiff (a linear
    stand-in pair on the host): the all-reduced loss and gradient equal one
    pair over all 5 suns to FP64 summation order."""
    from tests.shard_models import LinearPair

    r = _run_ranks(None, None, tmp_path / "d.npz", argv=["diff", str(tmp_path / "d.npz")])
    H = 7
    suns = np.array([[0.1 * k, -1.0, 0.05 * k] for k in range(5)], np.float32)  # as ShardedDiff holds them
    one = LinearPair(suns, H)
    rng = np.random.default_rng(3)
    for k in range(5):
        one.set_target(rng.standard_normal(40), receiver=k)
    one.set_params(rng.standard_normal((H, 2)), rng.standard_normal((H, 2)))
    assert (int(r["begin"]), int(r["end"])) == (0, 3)
    assert float(r["loss"]) == pytest.approx(one.forward(), rel=1e-12)
    np.testing.assert_allclose(r["grad"], one.backward(), rtol=1e-12, atol=1e-12)
