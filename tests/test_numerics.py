"""Host-side checks of numeric identities the kernels rely on."""
import numpy as np


def _floats_around(x: float, ulps: int = 4096) -> np.ndarray:
    """Every float32 within `ulps` units in the last place of x, plus specials."""
    c = np.float32(x).view(np.int32)
    span = np.arange(-ulps, ulps + 1, dtype=np.int64)
    if x > 0:
        bits = (c + span).astype(np.int32)
    else:
        bits = (c - span).astype(np.int32)
    vals = bits.view(np.float32)
    extra = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-30, -1e-30], np.float32)
    rng = np.random.default_rng(0)
    rand = (rng.standard_normal(100000) * 10.0 ** rng.integers(-8, 3, 100000)).astype(np.float32)
    return np.concatenate([vals, extra, rand])


def test_float_comparisons_with_double_epsilon():
    # qm_below_eps / qm_above_neg_eps / qm_below_neg_eps (csrc/vecmath.h) decide
    # comparisons with the double 1e-5 in float; they must agree for every float.
    eps32 = np.float32(1e-5)
    for centre in (1e-5, -1e-5):
        x = _floats_around(centre)
        with np.errstate(invalid="ignore"):
            d = x.astype(np.float64)
            assert np.array_equal(d < 1e-5, x <= eps32)
            assert np.array_equal(d <= 1e-5, x <= eps32)
            assert np.array_equal(d > -1e-5, x >= -eps32)
            assert np.array_equal(d >= -1e-5, x >= -eps32)
            assert np.array_equal(d < -1e-5, x < -eps32)


def test_aim_smoothing_and_adam():
    """Host pieces of the aim optimisation (solarenergy_chier_b200/aim.py):
    the FP64 smoothing equals a direct double loop of the pair's separable
    Gaussian (rows wrapping on a cylinder, columns zero outside), and Adam's
    first step moves every coordinate by lr against the gradient's sign."""
    from solarenergy_chier_b200 import aim

    rng = np.random.default_rng(2)
    img = rng.random((9, 13))
    w = aim.gaussian_weights(1.5).astype(np.float64)
    r = len(w) - 1
    for wrap in (True, False):
        tmp = np.zeros_like(img)
        for y in range(9):
            for x in range(13):
                for k in range(-r, r + 1):
                    c = x + k
                    if wrap:
                        c %= 13
                    if 0 <= c < 13:
                        tmp[y, x] += w[abs(k)] * img[y, c]
        want = np.zeros_like(img)
        for y in range(9):
            for x in range(13):
                for k in range(-r, r + 1):
                    if 0 <= y + k < 9:
                        want[y, x] += w[abs(k)] * tmp[y + k, x]
        np.testing.assert_allclose(aim.gaussian_smooth(img, 1.5, wrap), want, rtol=1e-13)
    opt = aim.Adam((3,), lr=0.1)
    x = opt.step(np.zeros(3), np.array([2.0, -5.0, 1e-3]))
    np.testing.assert_allclose(x, [-0.1, 0.1, -0.1], rtol=1e-4)
    t = aim.smooth_target(np.outer(np.hanning(40), np.hanning(60)), seed=1)
    lit = t > 0
    assert t.max() / t[lit].mean() <= 2.0
