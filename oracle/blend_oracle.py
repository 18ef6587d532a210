"""CPU oracle of the reference's two-image composition -- TEST INFRASTRUCTURE ONLY.

Restates GPUPyStitch._blend_pair (pysift/core.py:3686-3714) with gain
compensation, _find_seam (3386-3472) with _dp_vertical_seam /
_dp_horizontal_seam (3286-3383), _multiband_blend (3495-3553: _gauss_down /
_gauss_up, 3475-3493) and the final paste of _stitch_pair (3794-3814), in
numpy + scipy.ndimage (the algorithms cupyx.scipy.ndimage implements).

Canonical choices where the reference's arithmetic is not reproducible
(the CUDA path implements the same definition):
  * gain: the overlap means come from order-free integer sums -- each value
    rounded to a multiple of 2^-24 (exact for uint8 images), summed in int64,
    scaled back in float64, divided by the count and rounded to float32; the
    reference takes numpy's float32 means (a sequential sum over the rows);
  * seam-mask blur: separable, the float32 kernel of _seam_kernel,
    BORDER_REFLECT_101, rows then columns, float64 sums rounded to float32
    after each pass; the reference calls cv2.GaussianBlur (SIMD float sums).
faithful=True runs those two steps exactly as the reference does (numpy
means, cv2.GaussianBlur) to measure how far the canonical form moves.
"""
import numpy as np
import scipy.ndimage as ndi


def _seam_kernel():
    """The 25 float32 taps exp(-x^2 / 18) / sum, x = -12..12 (the kernel
    cv2.GaussianBlur(sigmaX=3) builds)."""
    x = np.arange(25, dtype=np.float64) - 12.0
    t = np.exp((-0.5 / 9.0) * (x * x))
    return (t / t.sum()).astype(np.float32)


def _reflect101(i, n):
    i = np.abs(i)
    i = np.where(i >= n, 2 * n - 2 - i, i)
    return np.clip(i, 0, n - 1)


def seam_blur(x, faithful=False):
    """GaussianBlur(sigma=3) of a float32 (H, W) mask."""
    if faithful:
        import cv2
        return cv2.GaussianBlur(x, (0, 0), sigmaX=3.0)
    k = _seam_kernel().astype(np.float64)
    H, W = x.shape
    r = 12
    xi = x.astype(np.float64)[:, _reflect101(np.arange(-r, W + r), W)]
    rows = np.zeros((H, W), np.float64)
    for j in range(2 * r + 1):
        rows += k[j] * xi[:, j:j + W]
    rows = rows.astype(np.float32).astype(np.float64)[_reflect101(np.arange(-r, H + r), H), :]
    out = np.zeros((H, W), np.float64)
    for j in range(2 * r + 1):
        out += k[j] * rows[j:j + H, :]
    return out.astype(np.float32)


def canonical_mean(v):
    """Per-channel mean of the rows of v (n, 3) float32: values rounded to
    multiples of 2^-24, summed in int64, scaled back in float64, divided by n
    in float64, rounded to float32."""
    q = np.rint(v.astype(np.float64) * 16777216.0).astype(np.int64).sum(0)
    return ((q.astype(np.float64) / 16777216.0) / float(len(v))).astype(np.float32)


def gain_compensate(w1, c2, ov, faithful=False):
    """core.py:3692-3699 (color_match='gain')."""
    if not ov.any():
        return w1
    if faithful:
        m2 = c2[ov].mean(0)
        m1 = w1[ov].mean(0)
    else:
        m2 = canonical_mean(c2[ov])
        m1 = canonical_mean(w1[ov])
    gain = (m2 + np.float32(1e-3)) / (m1 + np.float32(1e-3))
    return np.clip(w1 * np.clip(gain, np.float32(0.5), np.float32(2.0)), 0, 255).astype(np.float32)


def seam_cost(w1, c2, ov):
    """The cost map of _find_seam (core.py:3411-3420), float32."""
    d = w1 - c2
    color = np.sqrt((d[:, :, 0] * d[:, :, 0] + d[:, :, 1] * d[:, :, 1]) + d[:, :, 2] * d[:, :, 2])
    s = (w1 + c2) * np.float32(0.5)
    avg = ((s[:, :, 0] + s[:, :, 1]) + s[:, :, 2]) / np.float32(3.0)
    gx = ndi.sobel(avg, axis=1)
    gy = ndi.sobel(avg, axis=0)
    cost = color + np.float32(0.05) * np.sqrt(gx * gx + gy * gy)
    cost = cost.astype(np.float32)
    cost[~ov] = np.float32(1e9)
    return cost


def dp_vertical(cost, ov):
    """_dp_vertical_seam (core.py:3286-3334)."""
    H, W = cost.shape
    INF = 1e18
    ov_rows = np.where(np.any(ov, axis=1))[0]
    if len(ov_rows) == 0:
        return np.zeros(H, np.int32)
    dp = np.full((H, W), INF, np.float64)
    bt = np.zeros((H, W), np.int32)
    r0 = ov_rows[0]
    dp[r0] = np.where(ov[r0], cost[r0].astype(np.float64), INF)
    prev_r = r0
    for r in ov_rows[1:]:
        prev = dp[prev_r]
        pl = np.empty(W); pl[0] = INF; pl[1:] = prev[:-1]
        pr = np.empty(W); pr[-1] = INF; pr[:-1] = prev[1:]
        stk = np.stack([pl, prev, pr])
        aidx = np.argmin(stk, axis=0)
        best = stk[aidx, np.arange(W)]
        dp[r] = np.where(ov[r], cost[r].astype(np.float64) + best, INF)
        bt[r] = np.clip(np.arange(W) + aidx - 1, 0, W - 1)
        prev_r = r
    r_last = ov_rows[-1]
    seam_c = int(np.argmin(np.where(ov[r_last], dp[r_last], INF)))
    seam = np.full(H, seam_c, np.int32)
    for i in range(len(ov_rows) - 1, 0, -1):
        seam[ov_rows[i - 1]] = bt[ov_rows[i], seam[ov_rows[i]]]
    return seam


def dp_horizontal(cost, ov):
    """_dp_horizontal_seam (core.py:3336-3383): the vertical DP on the transpose."""
    return dp_vertical(cost.T.copy(), ov.T.copy())


def find_seam(w1, c2, m1, m2, faithful=False):
    """_find_seam (core.py:3386-3472): float32 (H, W) seam mask, 1 = image 1."""
    H, W = m1.shape
    ov = m1 & m2
    seam = np.zeros((H, W), np.float32)
    seam[m1 & ~m2] = 1.0
    if not ov.any():
        return seam
    cost = seam_cost(w1, c2, ov)
    n_rows = int(np.any(ov, axis=1).sum())
    n_cols = int(np.any(ov, axis=0).sum())
    s1c = np.where(np.any(m1 & ~m2, axis=0))[0]
    s2c = np.where(np.any(m2 & ~m1, axis=0))[0]
    left = len(s1c) == 0 or len(s2c) == 0 or s1c.mean() <= s2c.mean()
    s1r = np.where(np.any(m1 & ~m2, axis=1))[0]
    s2r = np.where(np.any(m2 & ~m1, axis=1))[0]
    top = len(s1r) == 0 or len(s2r) == 0 or s1r.mean() <= s2r.mean()
    if n_rows >= n_cols:
        cols = dp_vertical(cost, ov)
        ovr = np.any(ov, axis=1)
        cc = np.arange(W)
        for r in range(H):
            if not ovr[r]:
                continue
            first = cc <= cols[r]
            v = np.where(first, 1.0 if left else 0.0, 0.0 if left else 1.0).astype(np.float32)
            seam[r] = np.where(ov[r], v, seam[r])
    else:
        rows = dp_horizontal(cost, ov)
        ovc = np.any(ov, axis=0)
        rr = np.arange(H)
        for c in range(W):
            if not ovc[c]:
                continue
            first = rr <= rows[c]
            v = np.where(first, 1.0 if top else 0.0, 0.0 if top else 1.0).astype(np.float32)
            seam[:, c] = np.where(ov[:, c], v, seam[:, c])
    blurred = seam_blur(seam, faithful)
    seam[ov] = blurred[ov]
    return seam


def gauss_down(x):
    """_gauss_down (core.py:3475-3483): gaussian_filter(sigma=1) per channel, [::2, ::2]."""
    out = np.stack([ndi.gaussian_filter(x[:, :, c], sigma=1.0) for c in range(x.shape[2])], axis=2)
    return out[::2, ::2]


def gauss_up(x, th, tw):
    """_gauss_up (core.py:3485-3493): zoom order 1 to (th, tw)."""
    return ndi.zoom(x, [th / x.shape[0], tw / x.shape[1], 1.0], order=1)


def multiband(I1, I2, seam, n_levels=6):
    """_multiband_blend (core.py:3495-3553)."""
    gm = np.repeat(seam[:, :, None], 3, axis=2)
    gp1, gp2, gpm = [I1], [I2], [gm]
    for _ in range(n_levels - 1):
        gp1.append(gauss_down(gp1[-1]))
        gp2.append(gauss_down(gp2[-1]))
        gpm.append(gauss_down(gpm[-1]))
    lp1, lp2 = [], []
    for k in range(n_levels - 1):
        th, tw = gp1[k].shape[:2]
        lp1.append(gp1[k] - gauss_up(gp1[k + 1], th, tw))
        lp2.append(gp2[k] - gauss_up(gp2[k + 1], th, tw))
    lp1.append(gp1[-1])
    lp2.append(gp2[-1])
    lpb = [gpm[k] * lp1[k] + (np.float32(1.0) - gpm[k]) * lp2[k] for k in range(n_levels)]
    res = lpb[-1]
    for k in range(n_levels - 2, -1, -1):
        th, tw = lpb[k].shape[:2]
        res = gauss_up(res, th, tw) + lpb[k]
    return res.astype(np.float32)


def hist_match(src, ref, ov):
    """_hist_match (core.py:3591-3625): per channel, the CDFs of the overlap
    values of src and ref (integer bins, np.histogram), the LUT
    np.interp(cdf_src, cdf_ref, 0..255) and src mapped through it."""
    out = src.copy()
    bins = np.arange(257, dtype=np.float32)
    for c in range(3):
        s_cnt, _ = np.histogram(src[ov, c].clip(0, 255), bins=bins)
        r_cnt, _ = np.histogram(ref[ov, c].clip(0, 255), bins=bins)
        s_cdf = np.cumsum(s_cnt).astype(np.float64)
        r_cdf = np.cumsum(r_cnt).astype(np.float64)
        s_cdf /= s_cdf[-1] + 1e-8
        r_cdf /= r_cdf[-1] + 1e-8
        lut = np.interp(s_cdf, r_cdf, np.arange(256))
        out[:, :, c] = np.interp(src[:, :, c].ravel().clip(0, 255), np.arange(256), lut).reshape(src.shape[:2])
    return out.astype(np.float32)


def seam_rmse(w1_gained, m1, c2, m2):
    """_seam_rmse (core.py:3555-3562) of the gained image 1, exact: the
    uint8-truncated differences squared, summed as integers."""
    ov = m1 & m2
    if not ov.any():
        return float("nan")
    a = np.clip(w1_gained, 0, 255).astype(np.uint8)[ov].astype(np.int64)
    b = np.clip(c2, 0, 255).astype(np.uint8)[ov].astype(np.int64)
    d = a - b
    return float(np.sqrt((d * d).sum() / d.size))


def blend_core(w1, m1, c2, m2, n_levels=6, faithful=False, color_match="gain"):
    """_blend_pair (core.py:3686-3714) on float32 canvases: the blended float32
    image (before any clipping), the union mask and the seam RMSE.
    color_match 'hist' matches histograms, anything else applies the gain."""
    w1 = np.asarray(w1, np.float32)
    c2 = np.asarray(c2, np.float32)
    ov = m1 & m2
    if color_match == "hist":
        if ov.any():
            w1 = hist_match(w1, c2, ov)
    else:
        w1 = gain_compensate(w1, c2, ov, faithful)
    seam = find_seam(w1, c2, m1, m2, faithful)
    I1 = np.zeros_like(w1)
    I2 = np.zeros_like(w1)
    I1[m1] = w1[m1]
    I2[m2] = c2[m2]
    I1[~m1 & m2] = c2[~m1 & m2]
    I2[~m2 & m1] = w1[~m2 & m1]
    out = multiband(I1, I2, seam, n_levels)
    return out, m1 | m2, seam_rmse(w1, m1, c2, m2)


def paste(out, both):
    """The paste of _stitch_pair (core.py:3806-3809)."""
    pano = np.zeros(out.shape, np.uint8)
    pano[both] = np.clip(out[both], 0, 255).astype(np.uint8)
    return pano


def blend_pair(warped1, m1, canvas2, m2, n_levels=6, faithful=False, color_match="gain"):
    """_blend_pair + the paste of _stitch_pair: uint8 (H, W, 3) canvas (before
    the inner-rectangle crop) and the union mask."""
    out, both, _ = blend_core(warped1.astype(np.float32), m1, canvas2.astype(np.float32), m2, n_levels, faithful,
                              color_match)
    return paste(out, both), both


def compose3(warped1, m1, canvas2, m2, warped3, m3, n_levels=6, faithful=False, color_match="gain"):
    """The composition of _stitch_triple (core.py:3913-3953): image 1 blended
    with image 2, the float result blended with image 3 (gain on the float
    image, seam, multiband), paste.  Returns (pano uint8 before the crop,
    union mask, seam RMSE 1-2, seam RMSE 12-3)."""
    b12, m12, r12 = blend_core(warped1.astype(np.float32), m1, canvas2.astype(np.float32), m2, n_levels, faithful,
                               color_match)
    out, both, r23 = blend_core(b12, m12, warped3.astype(np.float32), m3, n_levels, faithful, color_match)
    return paste(out, both), both, r12, r23
