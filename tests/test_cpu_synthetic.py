"""The seeded synthetic inputs of the tests and the bench, on the CPU: the
same seed gives the same input, and each generator keeps the shapes, ranges
and structure its docstring states (the bench's workloads stand in for the
reference's datasets through them)."""
import math

import numpy as np
import pytest

from pysift_b200 import synthetic


def test_scene_is_seeded():
    a = synthetic.scene(120, 160, seed=3)
    assert a.shape == (120, 160) and a.dtype == np.uint8
    assert np.array_equal(a, synthetic.scene(120, 160, seed=3))
    assert not np.array_equal(a, synthetic.scene(120, 160, seed=4))
    assert 60 < a.mean() < 200 and a.std() > 5


@pytest.mark.parametrize("seed", range(8))
def test_random_homography_ranges(seed):
    W, H = 1280, 960
    Hm = synthetic.random_homography(np.random.default_rng(seed), W, H)
    assert Hm[2, 2] == 1.0
    # perspective terms of at most 1e-4, rotated, scaled by up to 1.1 and
    # renormalised by H[2,2] = 1 - p.c >= ~0.89
    assert np.all(np.abs(Hm[2, :2]) <= 1e-4 * 1.1 * math.sqrt(2) / 0.88)
    # at the view centre the perspective terms act on a zero vector, so the
    # map's Jacobian there is the rotation by at most 10 degrees, scaled by 0.9..1.1
    def proj(x, y):
        p = Hm @ np.array([x, y, 1.0])
        return p[:2] / p[2]

    e = 1e-3
    J = np.stack([(proj(W / 2 + e, H / 2) - proj(W / 2 - e, H / 2)) / (2 * e),
                  (proj(W / 2, H / 2 + e) - proj(W / 2, H / 2 - e)) / (2 * e)], axis=1)
    sc = math.sqrt(abs(np.linalg.det(J)))
    th = math.degrees(math.atan2(J[1, 0], J[0, 0]))
    assert 0.89 < sc < 1.11 and abs(th) < 10.5
    # the view centre moves left by 60-70 % of the width (30-40 % overlap)
    c = Hm @ np.array([W / 2, H / 2, 1.0])
    shift = c[0] / c[2] - W / 2
    assert -0.71 * W < shift < -0.59 * W


def test_stitch_pair_views_agree_under_the_true_homography():
    import cv2
    img1, img2, Hm = synthetic.stitch_pair(240, 320, seed=5)
    assert img1.shape == img2.shape == (240, 320, 3) and img1.dtype == np.uint8
    again = synthetic.stitch_pair(240, 320, seed=5)
    assert np.array_equal(img1, again[0]) and np.array_equal(img2, again[1])
    w1 = cv2.warpPerspective(img1.astype(np.float32), Hm, (320, 240), flags=cv2.INTER_LINEAR, borderValue=-1)
    ok = (w1 >= 0).all(-1)
    ok[:2] = ok[-2:] = False
    ok[:, :2] = ok[:, -2:] = False
    assert ok.mean() > 0.2
    diff = np.abs(w1[ok] - img2[ok].astype(np.float32))
    assert diff.mean() < 6.0


def test_descriptor_sets_half_noisy_copies():
    a, b = synthetic.descriptor_sets(64, 80, seed=2, D=128)
    assert a.shape == (64, 128) and b.shape == (80, 128) and a.dtype == b.dtype == np.uint8
    a2, b2 = synthetic.descriptor_sets(64, 80, seed=2, D=128)
    assert np.array_equal(a, a2) and np.array_equal(b, b2)
    linf = np.abs(b.astype(np.int32)[:, None, :] - a.astype(np.int32)[None, :, :]).max(-1)
    assert int((linf.min(1) <= 3).sum()) == 40
    assert 0 < a.mean() < 64 and a.max() < 255


def test_batch_and_pair_sizes():
    sizes = synthetic.batch_sizes(96, seed=0)
    assert len(sizes) == 96 and sizes == synthetic.batch_sizes(96, seed=0)
    assert all(360 <= h <= 3000 and 480 <= w <= 4000 for h, w in sizes)
    pairs = synthetic.pair_sizes(32, seed=0)
    assert len(pairs) == 32 and all(960 <= h <= 2000 and 1280 <= w <= 3000 for h, w in pairs)
