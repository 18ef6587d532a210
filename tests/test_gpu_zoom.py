"""2x cubic B-spline upsample (pysift_zoom2x_u8) against the oracle, bit for bit.

The device path is three kernels: a column FIR of the 61-tap spline
prefilter, an in-place row FIR that walks each row in chunks of 2048
outputs (the left halo of a chunk comes from a carry of the previous
chunk's inputs), and the 4x4 interpolation.  The shapes cover rows that fit
one chunk, rows that end exactly on a chunk boundary, rows whose last chunk
is narrower than the 30-tap halo (the mirrored right edge then reaches back
into the previous chunk), tall narrow images and one- and two-pixel edges.
The fp16 tier rounds the base image and the output to binary16.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 3), (7, 9), (3, 2048), (3, 2049), (2, 2077), (2, 2078), (4, 4096 + 29),
          (5, 6200), (2100, 3), (61, 37), (97, 2300)]


def _zoom_gpu(img, fp16):
    import torch
    from pysift_b200 import _lib
    lib = _lib.load()
    H, W = img.shape
    dev = torch.device("cuda", 0)
    g = torch.from_numpy(img).to(dev)
    coef = torch.full((H * W,), float("nan"), dtype=torch.float64, device=dev)
    pitch = 2 * W + 5
    out = torch.full((2 * H, pitch), float("nan"), dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.pysift_zoom2x_u8(g.data_ptr(), H, W, W, int(fp16), coef.data_ptr(), out.data_ptr(), pitch, st)
    assert rc == 0, lib.pysift_last_error()
    torch.cuda.synchronize(dev)
    got = out.cpu().numpy()
    assert np.isnan(got[:, 2 * W:]).all(), "wrote past the row"
    return got[:, :2 * W]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("fp16", [False, True])
def test_zoom2x_matches_oracle(shape, fp16, oracle_lib):
    from oracle import oracle
    rng = np.random.default_rng(shape[0] * 7919 + shape[1] + int(fp16))
    img = (rng.random(shape) * 256).astype(np.uint8)
    base = img.astype(np.float32) / np.float32(255.0)
    if fp16:
        base = base.astype(np.float16).astype(np.float32)
    ref = oracle.zoom2x(base)
    if fp16:
        ref = ref.astype(np.float16).astype(np.float32)
    got = _zoom_gpu(img, fp16)
    assert got.shape == ref.shape
    bad = np.argwhere(got.view(np.int32) != ref.view(np.int32))
    assert bad.size == 0, f"{len(bad)} differing pixels, first at {bad[:3].tolist()}"
