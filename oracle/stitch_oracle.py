"""CPU oracle for GPUPyStitch's two-image path -- TEST INFRASTRUCTURE ONLY.

Follows pysift/core.py:3720-3818: cv2 BGR->gray and CLAHE (the calls the
reference itself makes on this machine: kornia is absent), SIFT (the
OracleSIFT restatement with GPUPyStitch's n_octaves=4), stable top-k by
response, L2 + PCA-64 + fp16 mutual ratio test (oracle/match_oracle.py),
RANSAC/MAGSAC++ with LO refits (stitch_oracle.c), canvas, warp, the
reference's gain + seam + multiband composition (blend_oracle.py) or a feather
(stitch_oracle.c) and the reference's inner-rectangle crop.
"""
import ctypes

import numpy as np

from . import match_oracle
from .oracle import OracleSIFT, lib, _p


def _setup():
    L = lib()
    L.orc_ransac.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                             ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.orc_dlt.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    L.orc_l2_normalize.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_void_p]
    L.orc_pca_stats.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.orc_pca_basis.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.orc_pca_basis.restype = ctypes.c_int
    L.orc_pca_project.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_int, ctypes.c_void_p]
    L.orc_warp_feather.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_float,
                                   ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.orc_test_exp_d.restype = ctypes.c_double
    L.orc_test_exp_d.argtypes = [ctypes.c_double]
    return L


def mt19937_u32(seed, n):
    """Raw MT19937 stream (what torch.randint reduces modulo N on a CPU generator)."""
    rs = np.random.RandomState(seed)
    return rs.randint(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)


def ransac(p1, p2, n_hyp, thr, sigma_max, magsac=True, min_inliers=10, seed=42):
    L = _setup()
    p1 = np.ascontiguousarray(p1, np.float64)
    p2 = np.ascontiguousarray(p2, np.float64)
    n = len(p1)
    rnd = mt19937_u32(seed, 4 * n_hyp)
    H = np.zeros(9, np.float64)
    mask = np.zeros(n, np.uint8)
    info = np.zeros(3, np.int32)
    scores = np.zeros(n_hyp, np.float64)
    L.orc_ransac(_p(p1), _p(p2), n, _p(rnd), n_hyp, float(thr), float(sigma_max), 1 if magsac else 0, min_inliers,
                 _p(H), _p(mask), _p(info), _p(scores))
    return H.reshape(3, 3), mask.astype(bool), info, scores


def dlt(p1, p2):
    L = _setup()
    p1 = np.ascontiguousarray(p1, np.float64)
    p2 = np.ascontiguousarray(p2, np.float64)
    H = np.zeros(9, np.float64)
    L.orc_dlt(_p(p1), _p(p2), len(p1), _p(H))
    return H.reshape(3, 3)


def l2_normalize(d):
    L = _setup()
    d = np.ascontiguousarray(d, np.float32)
    out = np.empty_like(d)
    L.orc_l2_normalize(_p(d), d.shape[0], d.shape[1], _p(out))
    return out


def pca_stats(x):
    L = _setup()
    x = np.ascontiguousarray(x, np.float32)
    D = x.shape[1]
    mean = np.empty(D, np.float32)
    cov = np.empty((D, D), np.float64)
    L.orc_pca_stats(_p(x), x.shape[0], D, _p(mean), _p(cov))
    return mean, cov


def pca_basis(cov, P, return_sweeps=False):
    """(D, P) float32 basis of the P largest eigenvalues of the float64
    covariance by the canonical parallel Jacobi (stitch_oracle.c:
    orc_pca_basis; the reference takes cp.linalg.eigh, pysift/core.py:2734)."""
    L = _setup()
    cov = np.ascontiguousarray(cov, np.float64)
    D = cov.shape[0]
    out = np.empty((D, P), np.float32)
    sw = ctypes.c_int(0)
    if L.orc_pca_basis(_p(cov), D, P, _p(out), ctypes.byref(sw)) != 0:
        raise ValueError("pca_basis: D must be even and <= 128, 1 <= P <= D")
    return (out, sw.value) if return_sweeps else out


def pca_project(x, mean, proj):
    L = _setup()
    x = np.ascontiguousarray(x, np.float32)
    P = proj.shape[1]
    out = np.empty((x.shape[0], P), np.float32)
    L.orc_pca_project(_p(x), x.shape[0], x.shape[1], _p(np.ascontiguousarray(mean)), _p(np.ascontiguousarray(proj)),
                      P, _p(out))
    return out


def warp_feather(img1, img2, hinv32, cw, ch, ox, oy, iox, ioy, feather=True):
    L = _setup()
    img1 = np.ascontiguousarray(img1)
    img2 = np.ascontiguousarray(img2)
    out = np.zeros((ch, cw, 3), np.uint8)
    warped = np.zeros((ch, cw, 3), np.uint8)
    m1 = np.zeros((ch, cw), np.uint8)
    m2 = np.zeros((ch, cw), np.uint8)
    h = np.ascontiguousarray(np.asarray(hinv32, np.float32).ravel())
    L.orc_warp_feather(_p(img1), img1.shape[0], img1.shape[1], _p(img2), img2.shape[0], img2.shape[1], cw, ch, _p(h),
                       float(np.float32(ox)), float(np.float32(oy)), iox, ioy, 1 if feather else 0, _p(out),
                       _p(warped), _p(m1), _p(m2))
    return out, warped, m1.astype(bool), m2.astype(bool)


def canvas_size(shape1, shape2, H):
    h1, w1 = shape1[:2]
    h2, w2 = shape2[:2]
    c1 = np.array([[0, 0, 1], [w1, 0, 1], [w1, h1, 1], [0, h1, 1]], dtype=np.float64).T
    wc = H @ c1
    wc /= wc[2]
    ax = np.concatenate([wc[0], [0, w2, w2, 0]])
    ay = np.concatenate([wc[1], [0, 0, h2, h2]])
    ox = max(0.0, -ax.min())
    oy = max(0.0, -ay.min())
    return int(np.ceil(ax.max() + ox)) + 1, int(np.ceil(ay.max() + oy)) + 1, ox, oy


def autocrop(pano, both):
    """pysift/core.py:3627-3684 verbatim in numpy."""
    H, W = both.shape
    row_valid = np.any(both, axis=1)
    col_valid = np.any(both, axis=0)
    if not row_valid.any():
        return pano
    r0 = int(np.where(row_valid)[0][0]); r1 = int(np.where(row_valid)[0][-1])
    c0 = int(np.where(col_valid)[0][0]); c1 = int(np.where(col_valid)[0][-1])
    sub = both[r0:r1 + 1, c0:c1 + 1]
    nr, nc = sub.shape
    left = np.argmax(sub, axis=1); right = nc - 1 - np.argmax(sub[:, ::-1], axis=1)
    top = np.argmax(sub, axis=0); bot = nr - 1 - np.argmax(sub[::-1, :], axis=0)
    ic0, ic1 = int(left.max()), int(right.min())
    ir0, ir1 = int(top.max()), int(bot.min())
    if ic0 >= ic1 or ir0 >= ir1:
        return pano[r0:r1 + 1, c0:c1 + 1]
    return pano[r0 + ir0:r0 + ir1 + 1, c0 + ic0:c0 + ic1 + 1]


class OracleStitch:
    def __init__(self, ransac_iters=1500, inlier_thresh=5.0, match_ratio=0.75, max_keypoints=8000, pca_dims=64,
                 n_octaves=4, clahe_clip=2.0, clahe_tile=8, high_vram=True, blend="multiband", n_blend_levels=6,
                 int8_matching=False, color_match="gain"):
        self.color_match = color_match
        self.int8_matching = int8_matching
        self.blend = blend
        self.n_blend_levels = n_blend_levels
        self.ransac_iters = ransac_iters
        self.inlier_thresh = inlier_thresh
        self.match_ratio = match_ratio
        self.max_keypoints = max_keypoints
        self.pca_dims = pca_dims
        self.clahe_clip = clahe_clip
        self.clahe_tile = clahe_tile
        self.sift = OracleSIFT(n_octaves=n_octaves, high_vram=high_vram)
        self.pca = None

    def features(self, img):
        import cv2
        gray = cv2.cvtColor(img, cv2.COLOR_BGR2GRAY)
        gray = cv2.createCLAHE(clipLimit=self.clahe_clip, tileGridSize=(self.clahe_tile, self.clahe_tile)).apply(gray)
        r = self.sift.detect_and_compute(gray)
        n = len(r["x"])
        order = np.arange(n)
        if n > self.max_keypoints:
            order = np.array(sorted(range(n), key=lambda i: -float(r["response"][i])), np.int64)[:self.max_keypoints]
        pts = np.stack([r["x"], r["y"]], 1)[order]
        return pts, r["desc"][order], gray

    def prepare(self, d1, d2):
        both = np.concatenate([l2_normalize(d1), l2_normalize(d2)])
        if self.pca is None:
            mean, cov = pca_stats(both)
            self.pca = (mean, pca_basis(cov, self.pca_dims))
        p = pca_project(both, *self.pca)
        if not self.int8_matching:
            p = p.astype(np.float16)
        return p[:len(d1)], p[len(d1):]

    def stitch(self, img1, img2):
        pts1, d1, _ = self.features(img1)
        pts2, d2, _ = self.features(img2)
        a, b = self.prepare(d1, d2)
        if self.int8_matching:
            m = match_oracle.match_i8(a, b, self.match_ratio)   # pysift/core.py:2894-2923
        else:
            m = match_oracle.match_fp16(a, b, self.match_ratio)
        pairs = m["pairs"]
        p1 = pts1[pairs[:, 0]].astype(np.float64)
        p2 = pts2[pairs[:, 1]].astype(np.float64)
        H, mask, info, _ = ransac(p1, p2, self.ransac_iters, self.inlier_thresh, self.inlier_thresh)
        cw, ch, ox, oy = canvas_size(img1.shape, img2.shape, H)
        hinv = np.linalg.inv(H).astype(np.float32)
        iox, ioy = int(round(ox)), int(round(oy))
        out, warped, m1, m2 = warp_feather(img1, img2, hinv, cw, ch, ox, oy, iox, ioy)
        if self.blend == "multiband":
            from . import blend_oracle
            canvas2 = np.zeros((ch, cw, 3), np.uint8)
            ye, xe = min(ioy + img2.shape[0], ch), min(iox + img2.shape[1], cw)
            canvas2[ioy:ye, iox:xe] = img2[:ye - ioy, :xe - iox]
            out, _ = blend_oracle.blend_pair(warped, m1, canvas2, m2, self.n_blend_levels,
                                             color_match=self.color_match)
        pano = autocrop(out, m1 | m2)
        return dict(pano=pano, H=H, mask=mask, info=info, pairs=pairs, p1=p1, p2=p2, n1=len(pts1), n2=len(pts2),
                    canvas=out, canvas_size=(cw, ch), ox=ox, oy=oy)

    def stitch3(self, img1, img2, img3):
        """_stitch_triple (pysift/core.py:3820-3966) without depth: matches 1-2
        and 2-3 (PCA fitted on the first pair), RANSAC 1->2 and 3->2, the
        shared canvas, the two-pass composition (blend_oracle.compose3) and
        the crop."""
        from . import blend_oracle
        pts1, d1, _ = self.features(img1)
        pts2, d2, _ = self.features(img2)
        pts3, d3, _ = self.features(img3)
        ms = []
        for da, db in ((d1, d2), (d2, d3)):
            a, b = self.prepare(da, db)
            ms.append(match_oracle.match_i8(a, b, self.match_ratio) if self.int8_matching
                      else match_oracle.match_fp16(a, b, self.match_ratio))
        p12, p23 = ms[0]["pairs"], ms[1]["pairs"]
        pA, pB1 = pts1[p12[:, 0]].astype(np.float64), pts2[p12[:, 1]].astype(np.float64)
        pB2, pC = pts2[p23[:, 0]].astype(np.float64), pts3[p23[:, 1]].astype(np.float64)
        H12, _, info12, _ = ransac(pA, pB1, self.ransac_iters, self.inlier_thresh, self.inlier_thresh)
        H32, _, info32, _ = ransac(pC, pB2, self.ransac_iters, self.inlier_thresh, self.inlier_thresh)
        cw, ch, ox, oy = canvas_size3(img1.shape, img2.shape, img3.shape, H12, H32)
        iox, ioy = int(round(ox)), int(round(oy))
        _, w1, m1, m2 = warp_feather(img1, img2, np.linalg.inv(H12).astype(np.float32), cw, ch, ox, oy, iox, ioy)
        _, w3, m3, _ = warp_feather(img3, img2, np.linalg.inv(H32).astype(np.float32), cw, ch, ox, oy, iox, ioy)
        canvas2 = np.zeros((ch, cw, 3), np.uint8)
        ye, xe = min(ioy + img2.shape[0], ch), min(iox + img2.shape[1], cw)
        canvas2[ioy:ye, iox:xe] = img2[:ye - ioy, :xe - iox]
        pano, both, r12, r23 = blend_oracle.compose3(w1, m1, canvas2, m2, w3, m3, self.n_blend_levels,
                                                     color_match=self.color_match)
        return dict(pano=autocrop(pano, both), H12=H12, H32=H32, pairs12=p12, pairs23=p23, info12=info12,
                    info32=info32, rmse12=r12, rmse23=r23, canvas=(cw, ch))


def canvas_size3(shape1, shape2, shape3, H12, H32):
    """_compute_canvas_size_3 (pysift/core.py:3190-3208)."""
    h2, w2 = shape2[:2]
    xs, ys = [0.0, float(w2), float(w2), 0.0], [0.0, 0.0, float(h2), float(h2)]
    for shp, H in ((shape1, H12), (shape3, H32)):
        h, w = shp[:2]
        c = np.array([[0, 0, 1], [w, 0, 1], [w, h, 1], [0, h, 1]], dtype=np.float64).T
        wc = H @ c
        wc /= wc[2]
        xs.extend(wc[0].tolist())
        ys.extend(wc[1].tolist())
    ax, ay = np.array(xs), np.array(ys)
    ox, oy = max(0.0, -ax.min()), max(0.0, -ay.min())
    return int(np.ceil(ax.max() + ox)) + 1, int(np.ceil(ay.max() + oy)) + 1, ox, oy

