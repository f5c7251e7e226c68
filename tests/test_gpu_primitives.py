"""The tracer's own correctly rounded float primitives against CUDA's, on
every 32-bit input pattern (bit for bit): the production kernels call them in
place of the CUDA intrinsics, so their results must not change.
"""
import pytest

from solarenergy_chier_b200 import microbench

pytestmark = pytest.mark.gpu


def test_own_primitives_equal_cuda_on_every_input(cuda_device):
    names = ["rsqrt (series refinement vs __frsqrt_rn)", "rsqrt without the range test, on [2^-125, 2^125)",
             "a / height by the precomputed reciprocal (a, quotient in [2^-90, 2^90])", "cylinder u = a / height + 0.5 in [0, 1]",
             "sqrt from the reciprocal root, [2^-100, 2^126)", "Newton reciprocal, |x| in [2^-100, 2^100]",
             "Markstein division, 2^33 hashed pairs"]
    got = microbench.primitive_mismatches(len(names))
    assert got == [0] * len(names), dict(zip(names, got))
