"""The arithmetic behind the kernels' own correctly rounded square root and
division (csrc/vecmath.h: qm_sqrt_by_rsqrt, qm_div_markstein), restated in
numpy with every float operation rounded as the device rounds it (products
and FMAs formed exactly in extended precision, then rounded once to float)
and checked on the CPU against correctly rounded results:

  * Markstein's square-root iteration s' = RN(s + RN(x - s*s) * (y/2)),
    s = RN(x y), y = RN(1/sqrt(x)), on every float in [1, 4) -- every
    significand at both exponent parities; the iteration is invariant under
    x -> 4x away from the range ends, so this covers [2^-100, 2^126);
  * Markstein's division q' = RN(q + RN(a - b q) y), q = RN(a y),
    y = RN(1/b), on hashed pairs and on pairs whose quotient is close to a
    half-integer;
  * the cylinder's v scaled by the double product with 1/(2 pi) against the
    reference's double quotient, on every float in [0, pi].

The device functions themselves are checked against CUDA's on all 2^32
inputs by tests/test_gpu_primitives.py; this file needs no GPU.
"""
from fractions import Fraction

import numpy as np

L = np.longdouble


def rn(v):
    return np.asarray(v).astype(np.float32)


def fma(a, b, c):
    """RN(a * b + c) for float32 arrays: the product is exact in the 64-bit
    significand of longdouble, the sum too for the cancelling sums used here."""
    return rn(a.astype(L) * b.astype(L) + c.astype(L))


def exact_fma(a, b, c):
    return np.float32(float(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))))


def test_sqrt_from_the_correctly_rounded_reciprocal_root():
    assert np.finfo(L).nmant >= 63, "needs an extended-precision longdouble"
    bits = np.arange(np.float32(1.0).view(np.uint32), np.float32(4.0).view(np.uint32), dtype=np.uint32)
    x = bits.view(np.float32)
    y = rn(L(1) / np.sqrt(x.astype(L)))  # RN(1/sqrt(x)), double rounding below 2^-40
    s = x * y
    r = fma(-s, s, x)
    got = fma(r, np.float32(0.5) * y, s)
    want = np.sqrt(x.astype(np.float64)).astype(np.float32)  # RN(sqrt(x)): no double-rounding error for float
    bad = np.nonzero(got != want)[0]
    # confirm any apparent miss with exact rational arithmetic
    real = [i for i in bad if exact_fma(r[i], np.float32(0.5) * y[i], s[i]) != want[i]]
    assert not real, [hex(int(bits[i])) for i in real[:5]]


def test_markstein_division_with_the_correctly_rounded_reciprocal():
    rng = np.random.default_rng(7)
    n = 1 << 21
    a = (rng.integers(1 << 23, 1 << 24, n) * 2.0 ** rng.integers(-60, 40, n)).astype(np.float32)
    b = (rng.integers(1 << 23, 1 << 24, n) * 2.0 ** rng.integers(-50, 40, n)).astype(np.float32)
    a *= np.where(rng.random(n) < 0.5, -1, 1).astype(np.float32)
    b *= np.where(rng.random(n) < 0.5, -1, 1).astype(np.float32)
    # quotients near k + 1/2, where a wrong last correction would show
    k = rng.integers(0, 4096, n).astype(np.float32) + np.float32(0.5)
    a = np.concatenate([a, b * k])
    b = np.concatenate([b, b])
    y = rn(L(1) / b.astype(L))
    q = a * y
    r = fma(-b, q, a)
    got = fma(r, y, q)
    want = a / b  # float32 division: correctly rounded
    bad = np.nonzero(got != want)[0]
    real = [i for i in bad if exact_fma(r[i], y[i], q[i]) != want[i]]
    assert not real, [(float(a[i]), float(b[i])) for i in real[:5]]


def test_cylinder_v_by_product_equals_the_quotient():
    """The production builds scale the cylinder's arc cosine by the double
    product with 1/(2 pi) instead of dividing by 2 pi in double as the
    reference does (csrc/ray_geom.h); rounded to float the two agree on every
    float in [0, pi] (IEEE double arithmetic: the CPU's equals the GPU's)."""
    inv = 1.0 / (2 * np.pi)
    end = int(np.float32(np.pi).view(np.uint32)) + 1
    step = 1 << 24
    bad = 0
    for begin in range(0, end, step):
        a = np.arange(begin, min(begin + step, end), dtype=np.uint32).view(np.float32).astype(np.float64)
        bad += int(np.count_nonzero((a * inv).astype(np.float32) != (a / (2 * np.pi)).astype(np.float32)))
    assert bad == 0
