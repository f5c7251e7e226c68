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
