"""The allocation-free zoom entry point gives the same result as the
caller-scratch one.

pysift_zoom2x_u8_noalloc serves callers that cannot allocate device memory
where they call the library (for instance a plugin running inside a host
application that owns the whole device heap): its scratch is a fixed
file-scope device array instead of a caller buffer.  This test calls both
entry points through the C ABI on images in a row, the larger first, so
that a later, smaller call would read anything the earlier one left behind
past its own pixels, and requires bit-identical outputs, the same bar as the
other GPU parity tests.  It runs the largest accepted input (exactly the
scratch's 2^20 pixels) and checks that one row more is refused.  The file
is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _zoom_both(lib, img, dev):
    import torch
    H, W = img.shape
    g = torch.from_numpy(img).to(dev)
    coef = torch.empty(H * W, dtype=torch.float64, device=dev)
    pitch = ((2 * W + 31) // 32) * 32
    ref = torch.full((2 * H, pitch), -1.0, dtype=torch.float32, device=dev)
    out = torch.full((2 * H, pitch), -2.0, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.pysift_zoom2x_u8(g.data_ptr(), H, W, W, 0, coef.data_ptr(), ref.data_ptr(), pitch, st)
    assert rc == 0, lib.pysift_last_error()
    rc = lib.pysift_zoom2x_u8_noalloc(g.data_ptr(), H, W, W, 0, out.data_ptr(), pitch, st)
    assert rc == 0, lib.pysift_last_error()
    torch.cuda.synchronize(dev)
    return ref[:, :2 * W].cpu().numpy(), out[:, :2 * W].cpu().numpy()


def test_noalloc_zoom_matches_caller_scratch_twice():
    import torch
    from pysift_b200 import _lib
    from pysift_b200 import synthetic
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    # larger first: a stale read past the smaller call's H*W would show
    imgs = [synthetic.scene(480, 640, seed=22), synthetic.scene(300, 400, seed=21),
            synthetic.scene(37, 53, seed=23)]
    for img in imgs:
        ref, out = _zoom_both(lib, img, dev)
        assert np.array_equal(ref, out)
        assert np.isfinite(out).all() and out.max() > 0.0


def test_noalloc_zoom_largest_accepted_input():
    """1024 x 1024 = 2^20 pixels, the whole fixed scratch, twice in a row."""
    import torch
    from pysift_b200 import _lib
    from pysift_b200 import synthetic
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    assert 1024 * 1024 == _lib.ZOOM2X_NOALLOC_MAX_PIXELS
    for seed in (24, 25):
        ref, out = _zoom_both(lib, synthetic.scene(1024, 1024, seed=seed), dev)
        assert np.array_equal(ref, out)


def test_noalloc_zoom_rejects_oversized_input():
    import torch
    from pysift_b200 import _lib
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    H, W = 1025, 1024  # one row more than the fixed scratch holds
    assert H * W > _lib.ZOOM2X_NOALLOC_MAX_PIXELS
    g = torch.zeros((H, W), dtype=torch.uint8, device=dev)
    out = torch.empty((2 * H, 2 * W), dtype=torch.float32, device=dev)
    rc = lib.pysift_zoom2x_u8_noalloc(g.data_ptr(), H, W, W, 0, out.data_ptr(), 2 * W,
                                      torch.cuda.current_stream(dev).cuda_stream)
    assert rc == _lib.ERR_CAPACITY
    assert b"exceeds the fixed scratch" in lib.pysift_last_error()
