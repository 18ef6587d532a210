"""Seeded synthetic inputs for the SIFT / stitching workloads.

The reference's benchmark datasets (HPatches, IMC Phototourism, MegaDepth)
are not used; these generators stand in for them with the shapes, sizes and
value distributions the workloads are defined on:

* ``scene``: background 128, 50 axis-aligned rectangles (intensity
  U(30, 220)), 200 Gaussian blobs (sigma U(2, 25) px, amplitude U(-80, 80),
  centres uniform), band-limited noise (white N(0,1) blurred with sigma 1,
  rescaled to std 6), clipped to uint8.
* ``stitch_pair``: a colour scene (the generator per channel with gains
  U(0.8, 1.2)) seen by two views; view 2 is view 1 mapped by a homography
  with rotation U(+-10 deg), scale U(0.9, 1.1), a horizontal shift giving
  30-40 % overlap and perspective terms U(+-1e-4), plus N(0, 2) noise.
* ``descriptor_sets``: uint8 128-d descriptors from gamma(0.5) vectors,
  L2-normalised, clipped at 0.2, renormalised, x512, saturated; half of the
  second set are +-3-level noisy copies of the first.

All use ``numpy.random.Generator(PCG64(seed))``.
"""
import math

import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _blur1(img, sigma):
    r = int(4 * sigma + 0.5)
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    pad = np.pad(img, r, mode="reflect")
    tmp = np.zeros_like(pad)
    for i, w in enumerate(k):
        tmp += w * np.roll(pad, r - i, axis=1)
    out = np.zeros_like(pad)
    for i, w in enumerate(k):
        out += w * np.roll(tmp, r - i, axis=0)
    return out[r:-r, r:-r]


def scene_float(H, W, rng, n_blobs=200, n_rects=50):
    img = np.full((H, W), 128.0, np.float64)
    for _ in range(n_rects):
        h = int(rng.uniform(8, max(9, H / 4)))
        w = int(rng.uniform(8, max(9, W / 4)))
        y0 = int(rng.uniform(0, H - h))
        x0 = int(rng.uniform(0, W - w))
        img[y0:y0 + h, x0:x0 + w] = rng.uniform(30, 220)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    for _ in range(n_blobs):
        s = rng.uniform(2, 25)
        a = rng.uniform(-80, 80)
        cy, cx = rng.uniform(0, H), rng.uniform(0, W)
        r = int(4 * s + 1)
        y0, y1 = max(0, int(cy) - r), min(H, int(cy) + r + 1)
        x0, x1 = max(0, int(cx) - r), min(W, int(cx) + r + 1)
        if y0 >= y1 or x0 >= x1:
            continue
        d2 = (yy[y0:y1, x0:x1] - cy) ** 2 + (xx[y0:y1, x0:x1] - cx) ** 2
        img[y0:y1, x0:x1] += a * np.exp(-d2 / (2 * s * s))
    noise = _blur1(rng.standard_normal((H, W)), 1.0)
    noise *= 6.0 / max(noise.std(), 1e-12)
    return img + noise


def scene(H=480, W=640, seed=0):
    """Grayscale uint8 test image (640x480 by default)."""
    rng = _rng(seed)
    return np.clip(np.rint(scene_float(H, W, rng)), 0, 255).astype(np.uint8)


def random_homography(rng, W, H):
    """Rotation +-10 deg, scale 0.9-1.1, x-shift for 30-40 % overlap,
    perspective +-1e-4; maps view-1 pixel coordinates to view-2 ones."""
    th = math.radians(rng.uniform(-10, 10))
    sc = rng.uniform(0.9, 1.1)
    overlap = rng.uniform(0.30, 0.40)
    tx = -(1.0 - overlap) * W
    cx, cy = W / 2.0, H / 2.0
    C = np.array([[1, 0, -cx], [0, 1, -cy], [0, 0, 1]], np.float64)
    Ci = np.array([[1, 0, cx], [0, 1, cy], [0, 0, 1]], np.float64)
    R = np.array([[sc * math.cos(th), -sc * math.sin(th), 0],
                  [sc * math.sin(th), sc * math.cos(th), 0], [0, 0, 1]], np.float64)
    P = np.array([[1, 0, 0], [0, 1, 0], [rng.uniform(-1e-4, 1e-4), rng.uniform(-1e-4, 1e-4), 1]], np.float64)
    T = np.array([[1, 0, tx], [0, 1, 0], [0, 0, 1]], np.float64)
    Hm = T @ Ci @ P @ R @ C
    return Hm / Hm[2, 2]


def stitch_pair(H=960, W=1280, seed=0):
    """Two overlapping BGR uint8 views and the true view1->view2 homography."""
    import cv2
    rng = _rng(seed)
    Hm = random_homography(rng, W, H)
    # a scene wide enough to hold both views
    big_w = int(W * 2.2)
    big_h = int(H * 1.4)
    oy = (big_h - H) // 2
    chans = []
    gains = rng.uniform(0.8, 1.2, size=3)
    base = scene_float(big_h, big_w, rng, n_blobs=int(200 * 2.2 * 1.4), n_rects=int(50 * 2.2 * 1.4))
    for c in range(3):
        chans.append(base * gains[c])
    big = np.clip(np.stack(chans, -1), 0, 255).astype(np.float32)
    # view 1 = scene crop at (0, oy); view 2(u) = scene(S^-1 Hm^-1 u) with S the crop offset
    S = np.array([[1, 0, 0], [0, 1, -oy], [0, 0, 1]], np.float64)   # scene -> view1
    M2 = Hm @ S                                                      # scene -> view2
    v1 = big[oy:oy + H, :W]
    v2 = cv2.warpPerspective(big, M2, (W, H), flags=cv2.INTER_LINEAR, borderMode=cv2.BORDER_REFLECT)
    n1 = rng.normal(0, 2, size=v1.shape)
    n2 = rng.normal(0, 2, size=v2.shape)
    img1 = np.clip(np.rint(v1 + n1), 0, 255).astype(np.uint8)
    img2 = np.clip(np.rint(v2 + n2), 0, 255).astype(np.uint8)
    return img1, img2, Hm


def stitch_pair_fast(H=960, W=1280, seed=0):
    """stitch_pair with the cheaper scene_fast source scene (for large batches)."""
    import cv2
    rng = _rng(seed)
    Hm = random_homography(rng, W, H)
    big_w, big_h = int(W * 2.2), int(H * 1.4)
    oy = (big_h - H) // 2
    gains = rng.uniform(0.8, 1.2, size=3).astype(np.float32)
    base = scene_fast(big_h, big_w, seed=int(rng.integers(0, 2**31 - 1))).astype(np.float32)
    big = np.clip(base[:, :, None] * gains[None, None, :], 0, 255).astype(np.float32)
    S = np.array([[1, 0, 0], [0, 1, -oy], [0, 0, 1]], np.float64)
    M2 = Hm @ S
    v1 = big[oy:oy + H, :W]
    v2 = cv2.warpPerspective(big, M2, (W, H), flags=cv2.INTER_LINEAR, borderMode=cv2.BORDER_REFLECT)
    img1 = np.clip(np.rint(v1 + 2.0 * rng.standard_normal(v1.shape, dtype=np.float32)), 0, 255).astype(np.uint8)
    img2 = np.clip(np.rint(v2 + 2.0 * rng.standard_normal(v2.shape, dtype=np.float32)), 0, 255).astype(np.uint8)
    return img1, img2, Hm


def stitch_triple(H=480, W=640, seed=0):
    """Three overlapping BGR uint8 views (left, centre, right) of one scene and
    the true homographies view1 -> view2 and view3 -> view2 (view 2, the
    centre, is the reference frame of a three-image stitch)."""
    import cv2
    rng = _rng(seed)
    Ha = random_homography(rng, W, H)          # view1 -> view2
    Hb = random_homography(rng, W, H)          # view2 -> view3
    big_w, big_h = int(W * 2.9), int(H * 1.5)
    oy = (big_h - H) // 2
    gains = rng.uniform(0.8, 1.2, size=3).astype(np.float32)
    base = scene_fast(big_h, big_w, seed=int(rng.integers(0, 2**31 - 1))).astype(np.float32)
    big = np.clip(base[:, :, None] * gains[None, None, :], 0, 255).astype(np.float32)
    S = np.array([[1, 0, 0], [0, 1, -oy], [0, 0, 1]], np.float64)   # scene -> view1
    v1 = big[oy:oy + H, :W]
    v2 = cv2.warpPerspective(big, Ha @ S, (W, H), flags=cv2.INTER_LINEAR, borderMode=cv2.BORDER_REFLECT)
    v3 = cv2.warpPerspective(big, Hb @ Ha @ S, (W, H), flags=cv2.INTER_LINEAR, borderMode=cv2.BORDER_REFLECT)
    imgs = [np.clip(np.rint(v + 2.0 * rng.standard_normal(v.shape, dtype=np.float32)), 0, 255).astype(np.uint8)
            for v in (v1, v2, v3)]
    H32 = np.linalg.inv(Hb)
    return imgs[0], imgs[1], imgs[2], Ha, H32 / H32[2, 2]


def pair_sizes(n=32, seed=0):
    """Uneven stitch-pair sizes between 1280x960 and 3000x2000 (aspect 4:3 or 3:2)."""
    rng = _rng(seed + 7)
    out = []
    for _ in range(n):
        ah, aw = ((3, 4), (2, 3))[int(rng.integers(0, 2))]
        w = int(rng.uniform(1280, 3000))
        h = max(960, min(2000, int(round(w * ah / aw))))
        out.append((h, w))
    return out


def batch_pairs(n=32, seed=0):
    """n seeded BGR view pairs with the sizes of pair_sizes(n, seed)."""
    return [stitch_pair_fast(h, w, seed=seed * 1000 + i)[:2] for i, (h, w) in enumerate(pair_sizes(n, seed))]


def descriptor_sets(N=8192, M=8192, seed=0, D=128):
    """uint8 descriptor sets (N,D), (M,D); half of set 2 are noisy copies."""
    rng = _rng(seed)

    def make(n):
        v = rng.gamma(0.5, size=(n, D))
        v /= np.linalg.norm(v, axis=1, keepdims=True) + 1e-12
        v = np.minimum(v, 0.2)
        v /= np.linalg.norm(v, axis=1, keepdims=True) + 1e-12
        return np.clip(np.rint(v * 512.0), 0, 255).astype(np.uint8)

    a = make(N)
    b = make(M)
    h = min(M // 2, N)
    src = rng.permutation(N)[:h]
    dst = rng.permutation(M)[:h]
    noisy = a[src].astype(np.int32) + rng.integers(-3, 4, size=(h, D))
    b[dst] = np.clip(noisy, 0, 255).astype(np.uint8)
    return a, b


def batch_sizes(n=96, seed=0):
    """Uneven image sizes between 480x360 and 4000x3000, aspect 4:3, 3:2, 16:9."""
    rng = _rng(seed)
    aspects = [(4, 3), (3, 2), (16, 9)]
    out = []
    for _ in range(n):
        aw, ah = aspects[int(rng.integers(0, 3))]
        w = int(rng.uniform(480, 4000))
        h = int(round(w * ah / aw))
        h = max(360, min(3000, h))
        out.append((h, w))
    return out


def scene_fast(H, W, seed=0):
    """A cheaper scene for large batches: the blob/rectangle scene drawn at a
    quarter of the resolution (blob sigmas scaled with it), cubic-upsampled,
    plus band-limited noise at full resolution (sigma 1 blur, std 6)."""
    import cv2
    rng = _rng(seed)
    h, w = max(8, H // 4), max(8, W // 4)
    base = np.zeros((h, w), np.float64) + 128.0
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    for _ in range(50):
        x0, x1 = sorted(rng.integers(0, w, size=2))
        y0, y1 = sorted(rng.integers(0, h, size=2))
        base[y0:y1 + 1, x0:x1 + 1] = rng.uniform(30, 220)
    for _ in range(200):
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        s = rng.uniform(2, 25) / 4.0
        a = rng.uniform(-80, 80)
        r = int(3 * s) + 1
        ya, yb = max(0, int(cy) - r), min(h, int(cy) + r + 1)
        xa, xb = max(0, int(cx) - r), min(w, int(cx) + r + 1)
        if ya >= yb or xa >= xb:
            continue
        d2 = (yy[ya:yb, xa:xb] - cy) ** 2 + (xx[ya:yb, xa:xb] - cx) ** 2
        base[ya:yb, xa:xb] += a * np.exp(-d2 / (2 * s * s))
    img = cv2.resize(base.astype(np.float32), (W, H), interpolation=cv2.INTER_CUBIC)
    noise = cv2.GaussianBlur(rng.standard_normal((H, W)).astype(np.float32), (0, 0), 1.0)
    noise *= 6.0 / max(float(noise.std()), 1e-12)
    return np.clip(np.rint(img + noise), 0, 255).astype(np.uint8)


def batch_images(n=96, seed=0):
    """n seeded uint8 scenes with the uneven sizes of batch_sizes(n, seed)."""
    return [scene_fast(h, w, seed=seed * 1000 + i) for i, (h, w) in enumerate(batch_sizes(n, seed))]


def dense_texture(H, W, seed=0, sigma=2.0):
    """Band-limited noise texture (white noise blurred with `sigma`, std 40
    around 128): thousands of extrema per megapixel, used to exercise the
    keypoint cap and candidate truncation."""
    rng = _rng(seed)
    n = _blur1(rng.standard_normal((H, W)), sigma)
    n = n / max(n.std(), 1e-12) * 40 + 128
    return np.clip(np.rint(n), 0, 255).astype(np.uint8)
