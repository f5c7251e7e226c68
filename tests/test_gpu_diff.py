"""Differentiable forward / adjoint (qmcrt_fwd / qmcrt_bwd) against central
finite differences under common random numbers (the scene's fixed pools and
facet offsets), on the GPU.

Bar (written here): central differences with h = 1e-3 m for aim offsets
and 1e-5 rad for normal offsets, every heliostat of a 24-heliostat field
(100-730 m from the tower), relative error in the 2-norm per parameter kind:
  * heliostats within 450 m: normal offsets <= 1e-2, aim offsets <= 2e-2;
  * the whole field: <= 3e-2.
Measured on a B200: 0.21 % / 1.06 % within 450 m, 1.44 % / 1.57 % over the
field.  What separates the adjoint from the differences is the receiver's
edges: far heliostats' spots spill over the cylinder's silhouette and its
first and last rows, whose boundary terms the adjoint estimates from bands
of rays (per-heliostat ratios are printed).  The forward's total deposited
flux must equal the FP64 receiver power of the same rays.
"""
import numpy as np
import pytest

import solarenergy_chier_b200 as q
from solarenergy_chier_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def field(tmp_path_factory, cuda_device):
    return synth.large_field(tmp_path_factory.mktemp("d1"), seed=8, num_heliostats=24, helio_pixel=0.1,
                             receiver_pixel=0.05, groups=4, per_group=256)


def make(field, sigma=2.0):
    s = q.Scene(field.scene, field.config, device=0, seed=5)
    d = q.Diff(s, sigma)
    return s, d


def test_forward_conserves_energy(field):
    s, d = make(field)
    d.set_target(np.zeros((s.receiver(0)["height"], s.receiver(0)["width"]), np.float32))
    loss = d.forward()
    flux = d.flux(0).astype(np.float64)
    assert loss == pytest.approx(float((flux ** 2).sum()), rel=1e-4)
    # the same rays through the plain path: identical geometry and decisions
    s.trace(list(range(s.num_heliostats)))
    _, total = s.power()
    assert abs(flux.sum() - total) <= 2e-3 * total


def test_adjoint_matches_central_differences(field):
    s, d = make(field)
    H = s.num_heliostats
    rng = np.random.default_rng(3)
    aim = rng.uniform(-0.3, 0.3, (H, 2)).astype(np.float32)
    nrm = rng.uniform(-2e-4, 2e-4, (H, 2)).astype(np.float32)
    d.set_params(aim, nrm)
    d.set_target(np.zeros((s.receiver(0)["height"], s.receiver(0)["width"]), np.float32))
    d.forward()
    f0 = d.flux(0)
    target = np.roll(np.roll(f0, 6, axis=1), 3, axis=0) * np.float32(0.9)
    d.set_target(target)
    d.forward()
    grad = d.backward()
    ids = list(range(H))
    fd, ad = [], []
    for h in ids:
        for k in range(4):
            step = 1e-3 if k < 2 else 1e-5
            vals = []
            for sgn in (+1, -1):
                a, n = aim.copy(), nrm.copy()
                if k < 2:
                    a[h, k] += sgn * step
                else:
                    n[h, k - 2] += sgn * step
                d.set_params(a, n)
                vals.append(d.forward())
            fd.append((vals[0] - vals[1]) / (2 * step))
            ad.append(grad[h, k])
    fd, ad = np.array(fd).reshape(-1, 4), np.array(ad).reshape(-1, 4)
    for h, a, b in zip(ids, ad, fd):
        print(f"heliostat {h}: adjoint {a} finite differences {b} ratio {a / b}")
    dist = np.array([np.hypot(*s.heliostat(h)["pos"][[0, 2]]) for h in ids])
    # aim (m) and normal (rad) gradients have different scales: compare each kind
    failures = []
    for name, sel, bars in (("within 450 m", dist < 450.0, (2e-2, 1e-2)), ("whole field", dist > 0, (3e-2, 3e-2))):
        for cols, bar in zip(((0, 1), (2, 3)), bars):
            rel = np.linalg.norm(ad[sel][:, cols] - fd[sel][:, cols]) / np.linalg.norm(fd[sel][:, cols])
            print(f"relative error, {name}, parameters {cols}: {rel:.3e}")
            if rel > bar:
                failures.append(f"{name} {cols}: {rel:.3e} > {bar}")
    assert not failures, failures


def test_aim_optimisation_checked_by_the_plain_tracer(field):
    """Adam on the aim offsets from a perturbed start back toward the flux
    of the unperturbed field; every step re-traced by the plain tracer.
    Bars: both losses fall by more than half; the forward's and the plain
    tracer's FP64 powers agree to 1e-9 every step (the same hits); the
    plain tracer's smoothed flux is within 5 % L1 of the splatted flux."""
    from solarenergy_chier_b200 import aim

    s, d = make(field)
    d.set_light_range(0, 64)
    H = s.num_heliostats
    d.set_params()
    d.set_target(np.zeros((s.receiver(0)["height"], s.receiver(0)["width"]), np.float32))
    d.forward()
    target = d.flux(0)
    d.set_target(target)
    rng = np.random.default_rng(3)
    res = aim.optimise_aim(d, target, steps=25, lr_aim=0.05, aim0=rng.uniform(-0.5, 0.5, (H, 2)), check=True)
    h = res.history
    assert h[-1]["loss"] < 0.5 * h[0]["loss"]
    assert h[-1]["plain_loss"] < 0.5 * h[0]["plain_loss"]
    for r in h:
        assert abs(r["power"] - r["plain_power"]) <= 1e-9 * r["plain_power"], r
        assert r["plain_vs_splat_l1"] <= 0.05, r
    assert np.all(np.abs(res.aim) <= 1.0)


def test_plain_trace_keeps_the_adjoint_valid(field):
    s, d = make(field)
    d.set_light_range(0, 32)
    H = s.num_heliostats
    rng = np.random.default_rng(4)
    d.set_params(rng.uniform(-0.3, 0.3, (H, 2)), rng.uniform(-3e-4, 3e-4, (H, 2)))
    d.set_target(np.zeros((s.receiver(0)["height"], s.receiver(0)["width"]), np.float32))
    d.forward()
    g0 = d.backward()
    d.forward()
    d.plain()
    np.testing.assert_allclose(d.backward(), g0, rtol=1e-12, atol=1e-12 * np.abs(g0).max())


def test_recomputed_hit_records_give_the_checkpointed_gradient(field):
    """The adjoint with hit records recomputed segment by segment (a hit-bit
    trace before each adjoint launch) equals the one with the forward's
    checkpointed records, up to the order of the FP64 gradient atomics."""
    s, d = make(field)
    d.set_light_range(0, 48)
    H = s.num_heliostats
    rng = np.random.default_rng(6)
    d.set_params(rng.uniform(-0.3, 0.3, (H, 2)), rng.uniform(-3e-4, 3e-4, (H, 2)))
    d.set_target(np.zeros((s.receiver(0)["height"], s.receiver(0)["width"]), np.float32))
    d.set_hit_records(1)
    l1 = d.forward()
    assert d.hit_records()[0] is False and d.hit_records()[1] > 0
    g1 = d.backward()
    for seg in (256 * 7, 1 << 16, 0):
        d.set_hit_records(2, seg)
        l2 = d.forward()
        assert d.hit_records() == (True, 0)
        g2 = d.backward()
        assert l2 == pytest.approx(l1, rel=1e-12)
        np.testing.assert_allclose(g2, g1, rtol=1e-9, atol=1e-12 * np.abs(g1).max())
    d.set_hit_records(0)
    d.forward()
    assert d.hit_records()[0] is False  # a small field: checkpointing fits
    with pytest.raises(q.QmcrtError):
        d.set_hit_records(3)


def test_several_suns_in_one_pair(field):
    """One pair over two suns equals the sum of two one-sun pairs: loss,
    gradient (parameters shared by the suns), powers; receiver k = sun k."""
    s = q.Scene(field.scene, field.config, device=0, seed=5)
    suns = np.array([[0.0, -0.866, -0.5], [0.35, -0.75, 0.56]], np.float32)
    H = s.num_heliostats
    rng = np.random.default_rng(9)
    aim, nrm = rng.uniform(-0.3, 0.3, (H, 2)), rng.uniform(-3e-4, 3e-4, (H, 2))
    shape = (s.receiver(0)["height"], s.receiver(0)["width"])
    targets = [np.full(shape, 50.0 * (k + 1), np.float32) for k in range(2)]
    both = q.Diff(s, 2.0, suns=suns)
    assert both.num_suns == 2
    both.set_light_range(0, 32)
    both.set_params(aim, nrm)
    for k in range(2):
        both.set_target(targets[k], receiver=k)
    loss = both.forward()
    grad = both.backward()
    per, total = both.power()
    want_loss, want_grad, want_per = 0.0, np.zeros((H, 4)), np.zeros(H)
    for k in range(2):
        one = q.Diff(s, 2.0, suns=suns[k:k + 1])
        one.set_light_range(0, 32)
        one.set_params(aim, nrm)
        one.set_target(targets[k])
        want_loss += one.forward()
        want_grad += one.backward()
        want_per += one.power()[0]
        np.testing.assert_allclose(both.flux(k), one.flux(0), rtol=1e-5, atol=1e-6 * one.flux(0).max())
        one.close()
    assert loss == pytest.approx(want_loss, rel=1e-6)
    np.testing.assert_allclose(grad, want_grad, rtol=1e-6, atol=1e-9 * np.abs(want_grad).max())
    np.testing.assert_allclose(per, want_per, rtol=1e-12)
    assert total == pytest.approx(want_per.sum(), rel=1e-12)
    with pytest.raises(q.QmcrtError):
        both.flux(2)
    # one sun given explicitly equals the scene's own sun
    own = q.Diff(s, 2.0, suns=np.array(s.info.sun_dir[:], np.float32)[None])
    ref = q.Diff(s, 2.0)
    for x in (own, ref):
        x.set_light_range(0, 16)
        x.set_target(targets[0])
    assert own.forward() == pytest.approx(ref.forward(), rel=1e-12)


def test_aim_gradient_against_a_wider_difference_step(field):
    """The aim offsets' 1 % gap at h = 1e-3 m is the differences' own float
    noise: 1 mm moves a heliostat's normal by only ~2e-6 rad, six times less
    than the 1e-5 rad normal step, so the float rounding of the traced rays
    weighs six times more in the difference.  With h = 5e-3 m the same
    adjoint agrees with the central differences to within 1e-2 over the
    heliostats within 450 m (bar written here), and the two difference
    steps differ from each other by about as much as the adjoint differs
    from the narrow one."""
    s, d = make(field)
    H = s.num_heliostats
    rng = np.random.default_rng(3)
    aim = rng.uniform(-0.3, 0.3, (H, 2)).astype(np.float32)
    nrm = rng.uniform(-2e-4, 2e-4, (H, 2)).astype(np.float32)
    d.set_params(aim, nrm)
    d.set_target(np.zeros((s.receiver(0)["height"], s.receiver(0)["width"]), np.float32))
    d.forward()
    f0 = d.flux(0)
    d.set_target(np.roll(np.roll(f0, 6, axis=1), 3, axis=0) * np.float32(0.9))
    d.forward()
    grad = d.backward()[:, :2]

    def fd(step):
        out = np.zeros((H, 2))
        for h in range(H):
            for k in range(2):
                vals = []
                for sgn in (+1, -1):
                    a = aim.copy()
                    a[h, k] += sgn * step
                    d.set_params(a, nrm)
                    vals.append(d.forward())
                out[h, k] = (vals[0] - vals[1]) / (2 * step)
        return out

    narrow, wide = fd(1e-3), fd(5e-3)
    dist = np.array([np.hypot(*s.heliostat(h)["pos"][[0, 2]]) for h in range(H)])
    near = dist < 450.0

    def rel(a, b):
        return float(np.linalg.norm(a[near] - b[near]) / np.linalg.norm(b[near]))

    print(f"aim, within 450 m: adjoint vs h=1e-3 {rel(grad, narrow):.3e}, adjoint vs h=5e-3 {rel(grad, wide):.3e}, "
          f"h=1e-3 vs h=5e-3 {rel(narrow, wide):.3e}")
    assert rel(grad, wide) <= 1e-2


def test_adjoint_on_a_slice_of_the_benchmark_field(tmp_path, cuda_device):
    """The differentiation configuration on the benchmark field itself: every
    13th heliostat of the 624-heliostat field (48, spread over 100-750 m, the
    same grid), 0.02 m micro-facets (300,664 per heliostat), the 1257 x 600
    cylinder image, Gaussian splat sigma 2 px, a smooth seeded target with
    peak/mean <= 2, aim offsets U(+-1 m) and normal offsets U(+-1 mrad),
    central differences at h = 1e-3 m / 1e-5 rad under common random numbers
    (the scene's fixed pools and facet offsets), 256 light indexes per facet
    (3.7 G rays per forward, so the float rounding of the traced rays that
    the differences also difference averages out).

    Bars (written here): relative 2-norm error of the adjoint <= 1e-2 for
    both parameter kinds over the heliostats whose spots spill less than
    10 % of their rays past the receiver; over the heliostats within 450 m
    <= 1e-2 for the normal offsets and <= 2e-2 for the aim offsets; <= 3e-2
    for both over the slice.  Per heliostat the test prints the adjoint, the
    differences and the share of its rays that miss the receiver: the error
    follows that share (about 0.5 % below 10 % spill, 2-7 % at 20-50 %),
    i.e. the receiver's edges -- its silhouette and first and last rows,
    whose boundary terms the adjoint estimates from bands of rays --
    dominate it, not the float noise of the differences (64 and 256 lights
    give the same errors).
    """
    from solarenergy_chier_b200 import aim as aimmod

    files = synth.large_field(tmp_path, seed=0, keep_every=13)
    s = q.Scene(files.scene, files.config, device=0, seed=0)
    H = s.num_heliostats
    assert H == 48 and s.heliostat(0)["num_facets"] == 300664
    d = q.Diff(s, 2.0)
    d.set_light_range(0, 256)
    shape = (s.receiver(0)["height"], s.receiver(0)["width"])
    d.set_target(np.zeros(shape, np.float32))
    d.forward()
    target = aimmod.smooth_target(d.flux(0), seed=7)
    lit = target > 0
    assert target[lit].max() <= 2.0 * target[lit].mean() * 1.0001
    d.set_target(target)
    rng = np.random.default_rng(11)
    aim = rng.uniform(-1.0, 1.0, (H, 2)).astype(np.float32)
    nrm = rng.uniform(-1e-3, 1e-3, (H, 2)).astype(np.float32)
    d.set_params(aim, nrm)
    d.forward()
    grad = d.backward()
    fd = np.zeros((H, 4))
    for h in range(H):
        for k in range(4):
            step = 1e-3 if k < 2 else 1e-5
            vals = []
            for sgn in (+1, -1):
                a, n = aim.copy(), nrm.copy()
                if k < 2:
                    a[h, k] += sgn * step
                else:
                    n[h, k - 2] += sgn * step
                d.set_params(a, n)
                vals.append(d.forward())
            fd[h, k] = (vals[0] - vals[1]) / (2 * step)
    dist = np.array([np.hypot(*s.heliostat(h)["pos"][[0, 2]]) for h in range(H)])
    spills = np.zeros(H)
    for h in range(H):
        nf = s.heliostat(h)["num_facets"]
        codes = s.hit_records(h, nf // 2 - 1000, nf // 2 + 1000, 0, 64)
        spill = spills[h] = float(np.mean(codes == -3))
        rel = np.abs(grad[h] - fd[h]) / np.maximum(np.abs(fd[h]), 1e-30)
        print(f"heliostat {h} at {dist[h]:.0f} m, {100 * spill:.1f} % of rays miss the receiver: adjoint {grad[h]} "
              f"finite differences {fd[h]} relative {rel}")
    failures = []
    for name, sel, bars in (("spill under 10 %", spills < 0.1, (1e-2, 1e-2)),
                            ("within 450 m", dist < 450.0, (2e-2, 1e-2)), ("whole slice", dist > 0, (3e-2, 3e-2))):
        for cols, bar in zip(((0, 1), (2, 3)), bars):
            rel = np.linalg.norm(grad[sel][:, cols] - fd[sel][:, cols]) / np.linalg.norm(fd[sel][:, cols])
            print(f"relative error, {name}, parameters {cols}: {rel:.3e}")
            if rel > bar:
                failures.append(f"{name} {cols}: {rel:.3e} > {bar}")
    d.close()
    s.close()
    assert not failures, failures


def test_large_field_errors_against_fp64_on_a_subsample(tmp_path, cuda_device):
    """The large batched-adjoint configuration's rays against FP64 on a 1 %
    subsample: the 10,000-heliostat field (flat 10 x 10 m heliostats, 0.05 m
    micro-facets: 40,000 each, 150-1800 m, cylinder r 10 m x h 20 m at 200 m),
    every 100th heliostat x its 40,000 facets x light indexes 0-3 (1.6e7
    rays), at 2 of the 32 suns the large adjoint traces.  The plain tracer's
    rays are the forward's rays (the same hits: tests above), so their
    errors are the forward's.  Reported per sun: flux L1, per-heliostat and
    total power against the FP64 oracle, beside the reference's float
    arithmetic (the CPU oracle in float) on the same rays.  Bars (written
    here): the tracer within 1e-3 flux L1 and 1e-5 total power of the
    reference's float arithmetic, and no further from FP64 than it
    (1.05 x + 1e-4 in L1, + 2e-6 in power)."""
    import json

    from oracle import oracle

    files = synth.huge_field(tmp_path, seed=0)
    s = q.Scene(files.scene, files.config, device=0, seed=3)
    H = s.num_heliostats
    assert H == 10000 and s.heliostat(0)["num_facets"] == 40000
    ids = list(range(0, H, 100))
    dirs, pert = s.get_sample_pool()
    offsets = {h: s.get_facet_offsets(h) for h in ids}
    suns = synth.sun_positions()[::3][:32]
    lights = 4
    s.set_light_range(0, lights)
    for k in (0, 17):
        sun = suns[k]
        s.set_sun(sun)
        s.clear()
        s.clear_power()
        s.trace(ids)
        img = s.image(0).astype(np.float64)
        per, total = s.power()
        cfg = json.loads(files.config.read_text())
        cfg["sun_dir"] = [float(x) for x in sun]
        cpath = tmp_path / f"sun{k}.json"
        cpath.write_text(json.dumps(cfg))
        r32 = oracle.OracleScene.from_files(files.scene, cpath).trace(ids, dirs, pert, offsets, 0, lights)
        r64 = oracle.OracleScene.from_files(files.scene, cpath, precision=64).trace(ids, dirs, pert, offsets, 0,
                                                                                   lights)
        i32, i64 = r32["images"][0], r64["images"][0]
        t32, t64 = float(r32["power"].sum()), float(r64["power"].sum())
        assert t64 > 0

        def l1(a, b):
            return float(np.abs(a - b).sum() / b.sum())

        sel = np.array(ids)
        rep = {"sun": k, "rays": r32["counters"]["rays"], "flux_l1_vs_fp64": l1(img, i64),
               "reference_arithmetic_flux_l1_vs_fp64": l1(i32, i64), "flux_l1_vs_reference_arithmetic": l1(img, i32),
               "power_rel_vs_fp64": abs(total - t64) / t64,
               "reference_arithmetic_power_rel_vs_fp64": abs(t32 - t64) / t64,
               "max_heliostat_power_rel_vs_fp64": float(np.max(np.abs(per[sel] - r64["power"][sel]) /
                                                               np.maximum(r64["power"][sel], 1e-30)))}
        print("large field, 1 % subsample:", json.dumps(rep))
        assert rep["flux_l1_vs_reference_arithmetic"] <= 1e-3
        assert abs(total - t32) <= 1e-5 * t32
        assert rep["flux_l1_vs_fp64"] <= 1.05 * rep["reference_arithmetic_flux_l1_vs_fp64"] + 1e-4
        assert rep["power_rel_vs_fp64"] <= rep["reference_arithmetic_power_rel_vs_fp64"] + 2e-6
    s.close()
