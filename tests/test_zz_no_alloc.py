"""qmcrt_smooth_static: the trimmed-mean smoother that allocates no device memory.

Callers that may not call cudaMalloc - code running under a fixed
device-memory budget that another allocator has already reserved, or a
real-time loop that cannot take an allocation's latency or failure - smooth
their images with qmcrt_smooth_static, which keeps its image copy in a
static 16 MiB device array instead of allocating one.  These checks call it
through the C ABI and compare it with qmcrt_smooth on the same images, on
two calls in a row (the array keeps the previous call's contents), and check
that it refuses images beyond the array and leaves free device memory
unchanged.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import solarenergy_chier_b200 as q

pytestmark = pytest.mark.gpu

MAX_PIXELS = 4194304


def _images(shape, seed):
    rng = np.random.default_rng(seed)
    img = (rng.random(shape) * 100).astype(np.float32)
    img[rng.random(shape) < 0.3] = 0.0
    return img


def _smooth(fn, img, radius, ratio, stream=None):
    import torch

    t = torch.from_numpy(img.copy()).cuda()
    torch.cuda.synchronize()
    handle = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = fn(ctypes.c_void_p(t.data_ptr()), img.shape[1], img.shape[0], radius, ratio, handle)
    torch.cuda.synchronize()
    return rc, t.cpu().numpy()


def test_static_smoother_matches_allocating_smoother_twice():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("needs a CUDA device")
    lib = q.load()
    cases = [((600, 1257), 1, 0.17, 1), ((97, 131), 5, 0.05, 2)]
    for shape, radius, ratio, seed in cases:
        img = _images(shape, seed)
        rc_a, want = _smooth(lib.qmcrt_smooth, img, radius, ratio)
        rc_b, got = _smooth(lib.qmcrt_smooth_static, img, radius, ratio)
        assert rc_a == 0 and rc_b == 0, lib.qmcrt_last_error()
        # same kernel on the same copy: identical, well inside the smoother tests' tolerance
        assert np.array_equal(got, want)


def test_static_smoother_with_large_heaps_on_a_side_stream():
    """Radius 5 with trim ratio 0.25 needs 62 KiB of heaps per 256-thread
    block, above the 48 KiB default (the launch raises the limit); the call
    runs on a non-default stream, twice, and matches qmcrt_smooth.  A radius
    whose heaps would need more than the 227 KiB a block can have is refused
    with an error status instead of a launch, and the image is left as it was."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("needs a CUDA device")
    lib = q.load()
    side = torch.cuda.Stream()
    for seed in (6, 7):
        img = _images((211, 173), seed)
        rc_a, want = _smooth(lib.qmcrt_smooth, img, 5, 0.25, side)
        rc_b, got = _smooth(lib.qmcrt_smooth_static, img, 5, 0.25, side)
        assert rc_a == 0 and rc_b == 0, lib.qmcrt_last_error()
        assert np.array_equal(got, want)
    img = _images((64, 64), 8)
    rc, out = _smooth(lib.qmcrt_smooth_static, img, 10, 0.3)
    assert rc == 3
    assert lib.qmcrt_last_error().startswith(b"trimmed mean:")
    assert np.array_equal(out, img)


def test_static_smoother_allocates_nothing_and_rejects_large_images():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("needs a CUDA device")
    lib = q.load()
    img = _images((120, 160), 3)
    _smooth(lib.qmcrt_smooth_static, img, 1, 0.17)  # first call: device address lookup
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for seed in (4, 5):
        rc, _ = _smooth(lib.qmcrt_smooth_static, _images((120, 160), seed), 1, 0.17)
        assert rc == 0
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    t = torch.zeros(MAX_PIXELS + 1, device="cuda")
    rc = lib.qmcrt_smooth_static(ctypes.c_void_p(t.data_ptr()), MAX_PIXELS + 1, 1, 1, 0.17, None)
    assert rc == 1
    assert b"exceeds the static scratch" in lib.qmcrt_last_error()
