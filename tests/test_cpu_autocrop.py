"""The inner-rectangle crop box (pysift_autocrop_box, a host function of the
C library) against the oracle's numpy crop (pysift/core.py:3627-3684) on
coverage masks with the cases the crop distinguishes: nothing covered, a
single pixel, lines with gaps, a coverage with no inner rectangle, and
random warped quadrilaterals."""
import numpy as np
import pytest


def _extents(both):
    """Per-row / per-column first and last covered pixel (INT32_MAX / -1 for
    an empty line), as pysift_mask_extents writes them."""
    H, W = both.shape
    big = np.iinfo(np.int32).max
    rows_any, cols_any = both.any(axis=1), both.any(axis=0)
    row_lo = np.where(rows_any, np.argmax(both, axis=1), big)
    row_hi = np.where(rows_any, W - 1 - np.argmax(both[:, ::-1], axis=1), -1)
    col_lo = np.where(cols_any, np.argmax(both, axis=0), big)
    col_hi = np.where(cols_any, H - 1 - np.argmax(both[::-1, :], axis=0), -1)
    return np.concatenate([row_lo, row_hi, col_lo, col_hi]).astype(np.int32)


def _box(lib, both):
    H, W = both.shape
    e = _extents(both)
    box = np.empty(5, dtype=np.int32)
    p = e.ctypes.data
    assert lib.pysift_autocrop_box(p, p + 4 * H, p + 8 * H, p + 8 * H + 4 * W, W, H, box.ctypes.data) == 0
    return box


def _masks():
    rng = np.random.default_rng(5)
    yield np.zeros((7, 9), bool)
    m = np.zeros((7, 9), bool); m[3, 4] = True; yield m
    m = np.zeros((8, 8), bool); m[2, :] = True; m[:, 5] = True; yield m      # a cross: no inner rectangle
    m = np.zeros((9, 11), bool); m[1:8, 2:10] = True; m[4, 5] = False; yield m
    m = np.zeros((10, 12), bool); m[2:9, 1:11] = True; m[5, :] = False; yield m  # an empty row inside
    for _ in range(40):
        H, W = int(rng.integers(5, 60)), int(rng.integers(5, 60))
        yy, xx = np.mgrid[0:H, 0:W]
        c = rng.uniform(0, 1, size=(4, 2)) * [W, H]
        quad = np.array([[c[0, 0] * 0.3, c[0, 1] * 0.3], [W - c[1, 0] * 0.3, c[1, 1] * 0.3],
                         [W - c[2, 0] * 0.3, H - c[2, 1] * 0.3], [c[3, 0] * 0.3, H - c[3, 1] * 0.3]])
        inside = np.ones((H, W), bool)
        for k in range(4):
            a, b = quad[k], quad[(k + 1) % 4]
            inside &= (b[0] - a[0]) * (yy - a[1]) - (b[1] - a[1]) * (xx - a[0]) >= 0
        yield inside | (rng.random((H, W)) < 0.01)


@pytest.mark.parametrize("i", range(45))
def test_autocrop_box_equals_the_oracle_crop(i):
    from oracle import stitch_oracle as so
    from pysift_b200 import _lib
    lib = _lib.load()
    both = list(_masks())[i]
    H, W = both.shape
    pano = np.arange(H * W * 3, dtype=np.int64).reshape(H, W, 3)
    x, y, w, h, kind = (int(v) for v in _box(lib, both))
    want = so.autocrop(pano, both)
    assert np.array_equal(pano[y:y + h, x:x + w], want)
    if not both.any():
        assert kind == 0 and (x, y, w, h) == (0, 0, W, H)


def test_autocrop_box_argument_checks():
    import ctypes
    from pysift_b200 import _lib
    lib = _lib.load()
    e = np.zeros(4, dtype=np.int32)
    box = np.empty(5, dtype=np.int32)
    assert lib.pysift_autocrop_box(None, None, None, None, 1, 1, box.ctypes.data) == -1
    p = e.ctypes.data
    assert lib.pysift_autocrop_box(p, p, p, p, 0, 1, box.ctypes.data) == -1
    fake = ctypes.c_void_p(256)
    assert lib.pysift_copy2d(fake, 4, fake, 8, 16, 2, None) == -1  # row wider than the destination pitch
