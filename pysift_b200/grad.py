"""Differentiable SIFT descriptors and warp + feather blend (autograd).

Two torch.autograd.Functions with hand-written CUDA forward and backward
kernels (csrc/grad.cu, C ABI pysift_desc_f32_* / pysift_blur_adjoint /
pysift_warp_f32_*):

* ``descriptors(img, keypoints, sift)``: float descriptors (L2 -> clip 0.2
  -> L2, before RootSIFT and quantisation) of fixed keypoints on a float32
  image in [0, 1] (no 2x upsampling).  Keypoint location, scale and
  orientation are constants; the gradient flows into the image through the
  descriptor histograms, the central-difference gradients, every Gaussian
  blur of the pyramid and the octave subsampling.  Pyramid levels are
  recomputed in backward, not stored.
* ``warp_blend(img1, img2, h8, geometry)``: the float warp of image 1 by a
  homography onto the canvas with image 2 placed and the linear feather
  blend where both cover; gradients for both images and the 8 homography
  parameters (H[2][2] = 1).

``descriptors_torch`` and ``warp_blend_torch`` restate both forwards in
plain torch ops (any dtype) as references for the gradient checks.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib


def _st():
    return torch.cuda.current_stream().cuda_stream


def pyramid_params(sift):
    """(n_octaves, S, base (weights, radius), increments [(weights, radius)]) of
    a PySIFT instance, for the non-doubled base."""
    cfg = sift._cfg
    S = cfg.n_scales

    def wr(idx):
        r = int(cfg.blur_radius[idx])
        return np.array([cfg.blur_weights[idx][j] for j in range(2 * r + 1)], np.float32), r

    return cfg.n_octaves, S, wr(1), [wr(2 + s) for s in range(S + 2)]


def _blur(x, w, r):
    """Production blur (pysift_gauss_blur) of a 2-D float32 CUDA tensor."""
    H, W = x.shape
    out = torch.empty_like(x)
    rc = _lib.load().pysift_gauss_blur(x.data_ptr(), x.stride(0), out.data_ptr(), out.stride(0), H, W,
                                       w.ctypes.data_as(ctypes.c_void_p), r, _st())
    _lib.check(rc, "pysift_gauss_blur")
    return out


def _blur_adjoint(g, w, r, accumulate_into=None):
    H, W = g.shape
    out = accumulate_into if accumulate_into is not None else torch.empty_like(g)
    tmp = torch.empty_like(g)
    wd = torch.from_numpy(w).to(g.device)
    rc = _lib.load().pysift_blur_adjoint(g.data_ptr(), g.stride(0), out.data_ptr(), out.stride(0), tmp.data_ptr(),
                                         tmp.stride(0), H, W, wd.data_ptr(), r,
                                         1 if accumulate_into is not None else 0, _st())
    _lib.check(rc, "pysift_blur_adjoint")
    return out


def _levels(x, n_oct, S, base, incs, top):
    """Gaussian levels 0..top of every octave (list of lists of tensors)."""
    levels = []
    cur = _blur(x, *base) if base[1] > 0 else x.clone()
    for o in range(n_oct):
        lv = [cur]
        for s in range(top):
            w, r = incs[s]
            lv.append(_blur(lv[-1], w, r) if r > 0 else lv[-1].clone())
        levels.append(lv)
        if o + 1 < n_oct:
            cur = lv[S][::2, ::2].contiguous()
            if min(cur.shape) < 8:
                break
    return levels


def keypoints_for_grad(sift, kpts, octave):
    """(x, y, size, angle) rows and octaves of a non-doubled detection ->
    (n, 5) float rows [octave, scale index, centre row, centre column, angle]."""
    cfg = sift._cfg
    if sift.double_image:
        raise ValueError("use a PySIFT(double_image=False) instance for differentiable descriptors")
    k = kpts.detach().cpu().numpy().astype(np.float64)
    o = np.asarray(octave.detach().cpu().numpy() if isinstance(octave, torch.Tensor) else octave).astype(np.int64)
    S = cfg.n_scales
    rows = []
    for i in range(k.shape[0]):
        sc = float(1 << int(o[i]))
        sizes = np.array([cfg.kp_size[0][int(o[i])][s] for s in range(S + 3)], np.float32)
        si = int(np.argmin(np.abs(sizes - np.float32(k[i, 2]))))
        rows.append([o[i], si, int(np.float32(k[i, 1]) / np.float32(sc)), int(np.float32(k[i, 0]) / np.float32(sc)),
                     k[i, 3]])
    return torch.tensor(np.array(rows, np.float64).reshape(-1, 5), dtype=torch.float64)


class _Descriptors(torch.autograd.Function):
    @staticmethod
    def forward(ctx, img, kps, sift):
        n_oct, S, base, incs = pyramid_params(sift)
        x = img.detach().contiguous().float()
        top = int(kps[:, 1].max().item()) if kps.shape[0] else 1
        top = max(top, S)
        levels = _levels(x, n_oct, S, base, incs, top)
        lib = _lib.load()
        n = kps.shape[0]
        desc = torch.zeros((n, 128), dtype=torch.float32, device=img.device)
        hist = torch.zeros((n, 128), dtype=torch.float32, device=img.device)
        groups = {}
        for i, (o, si) in enumerate(kps[:, :2].long().tolist()):
            groups.setdefault((o, si), []).append(i)
        for (o, si), idx in groups.items():
            G = levels[o][si]
            sel = torch.tensor(idx, dtype=torch.long)
            kp = kps[sel][:, 2:5].float().contiguous().to(img.device)
            ph = int(sift._cfg.desc_ph[si])
            d = torch.empty((len(idx), 128), dtype=torch.float32, device=img.device)
            h = torch.empty_like(d)
            _lib.check(lib.pysift_desc_f32_forward(G.data_ptr(), G.shape[0], G.shape[1], G.stride(0), kp.data_ptr(),
                                                   len(idx), ph, h.data_ptr(), d.data_ptr(), _st()),
                       "pysift_desc_f32_forward")
            dev_idx = sel.to(img.device)
            desc[dev_idx] = d
            hist[dev_idx] = h
        ctx.save_for_backward(img, hist)
        ctx.kps = kps
        ctx.sift = sift
        ctx.groups = groups
        return desc

    @staticmethod
    def backward(ctx, gdesc):
        img, hist = ctx.saved_tensors
        sift, kps, groups = ctx.sift, ctx.kps, ctx.groups
        n_oct, S, base, incs = pyramid_params(sift)
        x = img.detach().contiguous().float()
        top = max(int(kps[:, 1].max().item()) if kps.shape[0] else 1, S)
        levels = _levels(x, n_oct, S, base, incs, top)       # recomputed, not stored
        lib = _lib.load()
        grads = [[torch.zeros_like(G) for G in lv] for lv in levels]
        gdesc = gdesc.contiguous().float()
        for (o, si), idx in groups.items():
            G = levels[o][si]
            sel = torch.tensor(idx, dtype=torch.long)
            kp = kps[sel][:, 2:5].float().contiguous().to(img.device)
            ph = int(sift._cfg.desc_ph[si])
            dev_idx = sel.to(img.device)
            h = hist[dev_idx].contiguous()
            gd = gdesc[dev_idx].contiguous()
            gG = grads[o][si]
            _lib.check(lib.pysift_desc_f32_backward(G.data_ptr(), G.shape[0], G.shape[1], G.stride(0), kp.data_ptr(),
                                                    len(idx), ph, h.data_ptr(), gd.data_ptr(), gG.data_ptr(), _st()),
                       "pysift_desc_f32_backward")
        # adjoint of the level chain, highest octave first
        for o in range(len(levels) - 1, -1, -1):
            g = grads[o]
            for s in range(len(g) - 1, 0, -1):
                w, r = incs[s - 1]
                if r > 0:
                    _blur_adjoint(g[s], w, r, accumulate_into=g[s - 1])
                else:
                    g[s - 1] += g[s]
            if o > 0:
                grads[o - 1][S][::2, ::2] += g[0]
        g0 = grads[0][0]
        gx = _blur_adjoint(g0, *base) if base[1] > 0 else g0
        return gx.to(img.dtype), None, None


def descriptors(img, keypoints, sift):
    """Float descriptors (n, 128) of fixed keypoints ([octave, scale index,
    centre row, centre column, angle] rows) on a float32 CUDA image in [0, 1],
    differentiable with respect to the image."""
    return _Descriptors.apply(img, keypoints, sift)


# -- plain-torch reference -------------------------------------------------
def _reflect_index(n, r, device):
    i = torch.arange(-r, n + r, device=device)
    i = torch.where(i < 0, -i - 1, i)
    i = torch.where(i >= n, 2 * n - 1 - i, i)
    return i


def _blur_torch(x, w, r):
    if r == 0:
        return x
    wt = torch.as_tensor(w, dtype=x.dtype, device=x.device)
    H, W = x.shape
    xi = x[:, _reflect_index(W, r, x.device)]
    h = torch.nn.functional.conv1d(xi.reshape(H, 1, -1), wt.flip(0).reshape(1, 1, -1)).reshape(H, W)
    hi = h[_reflect_index(H, r, x.device), :]
    v = torch.nn.functional.conv1d(hi.t().reshape(W, 1, -1), wt.flip(0).reshape(1, 1, -1)).reshape(W, H).t()
    return v


def _desc_torch_level(G, kp, ph):
    dev, dt = G.device, G.dtype
    H, W = G.shape
    side = 2 * ph + 1
    ar = torch.arange(side * side, device=dev)
    r_off = (ar // side - ph).to(dt)
    c_off = (ar % side - ph).to(dt)
    r0 = kp[:, 0:1].to(torch.long).to(dev)
    c0 = kp[:, 1:2].to(torch.long).to(dev)
    ang = (kp[:, 2:3] * (math.pi / 180.0)).to(dt).to(dev)
    rr = r0 + r_off.long()
    cc = c0 + c_off.long()
    cos_a, sin_a = torch.cos(ang), torch.sin(ang)
    xr = cos_a * c_off - sin_a * r_off
    yr = sin_a * c_off + cos_a * r_off
    scale = 4.0 / (2.0 * ph)
    xb = xr * scale + 1.5
    yb = yr * scale + 1.5
    act = (rr >= 1) & (rr < H - 1) & (cc >= 1) & (cc < W - 1) & (xb >= -0.5) & (xb < 3.5) & (yb >= -0.5) & (yb < 3.5)
    rrc = rr.clamp(1, H - 2)
    ccc = cc.clamp(1, W - 2)
    dx = G[rrc, ccc + 1] - G[rrc, ccc - 1]
    dy = G[rrc + 1, ccc] - G[rrc - 1, ccc]
    m2 = dx * dx + dy * dy
    ok = act & (m2 > 0)
    mag = torch.sqrt(torch.where(ok, m2, torch.ones_like(m2))) * ok
    ori = (torch.atan2(dy, dx) - ang) * (180.0 / math.pi) + 360.0
    ori = torch.where(ori >= 360.0, ori - 360.0, ori)
    sigma_d = ph * 0.5657
    gw = torch.exp(-(xr * xr + yr * yr) / (2.0 * sigma_d * sigma_d + 1e-12))
    ob = ori * (8.0 / 360.0)
    oi0 = torch.floor(ob).detach()
    df = ob - oi0
    xi0 = torch.floor(xb).detach()
    yi0 = torch.floor(yb).detach()
    dxb, dyb = xb - xi0, yb - yi0
    xa, xc = xi0.clamp(0, 3).long(), (xi0 + 1).clamp(0, 3).long()
    ya, yc = yi0.clamp(0, 3).long(), (yi0 + 1).clamp(0, 3).long()
    o0 = torch.remainder(oi0.long(), 8)
    o1 = torch.remainder(oi0.long() + 1, 8)
    wm = mag * gw
    n = kp.shape[0]
    hist = torch.zeros((n, 128), dtype=dt, device=dev)
    rows = torch.arange(n, device=dev).unsqueeze(1).expand_as(rr)
    for yy, wy in ((ya, 1 - dyb), (yc, dyb)):
        for xx, wx in ((xa, 1 - dxb), (xc, dxb)):
            for oo, wo in ((o0, 1 - df), (o1, df)):
                val = (wy * wx * wo * wm) * ok
                hist.index_put_((rows, yy * 32 + xx * 8 + oo), val, accumulate=True)
    n1 = torch.sqrt((hist * hist).sum(1, keepdim=True) + 1e-14)
    t = torch.clamp(hist / n1, max=0.2)
    n2 = torch.sqrt((t * t).sum(1, keepdim=True) + 1e-14)
    return t / n2


def descriptors_torch(img, keypoints, sift):
    """descriptors() restated with plain torch ops (autograd; any dtype)."""
    n_oct, S, base, incs = pyramid_params(sift)
    top = max(int(keypoints[:, 1].max().item()), S)
    levels = []
    cur = _blur_torch(img, *base)
    for o in range(n_oct):
        lv = [cur]
        for s in range(top):
            lv.append(_blur_torch(lv[-1], *incs[s]))
        levels.append(lv)
        if o + 1 < n_oct:
            cur = lv[S][::2, ::2]
            if min(cur.shape) < 8:
                break
    out = torch.zeros((keypoints.shape[0], 128), dtype=img.dtype, device=img.device)
    groups = {}
    for i, (o, si) in enumerate(keypoints[:, :2].long().tolist()):
        groups.setdefault((o, si), []).append(i)
    for (o, si), idx in groups.items():
        sel = torch.tensor(idx, dtype=torch.long)
        d = _desc_torch_level(levels[o][si], keypoints[sel][:, 2:5], int(sift._cfg.desc_ph[si]))
        out = out.index_put((sel.to(img.device),), d)
    return out


# -- warp + feather blend ---------------------------------------------------
def canvas_geometry(img1_shape, img2_shape, H):
    """(cw, ch, ox, oy, iox, ioy) of the stitch canvas (pysift/core.py:3171-3187)."""
    h1, w1 = img1_shape[:2]
    h2, w2 = img2_shape[:2]
    c1 = np.array([[0, 0, 1], [w1, 0, 1], [w1, h1, 1], [0, h1, 1]], dtype=np.float64).T
    wc = H @ c1
    wc /= wc[2]
    ax = np.concatenate([wc[0], [0, w2, w2, 0]])
    ay = np.concatenate([wc[1], [0, 0, h2, h2]])
    ox = max(0.0, -ax.min())
    oy = max(0.0, -ay.min())
    cw, ch = int(np.ceil(ax.max() + ox)) + 1, int(np.ceil(ay.max() + oy)) + 1
    return cw, ch, float(ox), float(oy), int(round(ox)), int(round(oy))


def _h_from8(h8):
    return torch.cat([h8.double(), torch.ones(1, dtype=torch.float64, device=h8.device)]).reshape(3, 3)


class _WarpBlend(torch.autograd.Function):
    @staticmethod
    def forward(ctx, img1, img2, h8, geometry):
        cw, ch, ox, oy, iox, ioy = geometry
        Hm = _h_from8(h8.detach())
        Hinv = torch.linalg.inv(Hm)
        hinv = np.ascontiguousarray(Hinv.cpu().numpy().ravel().astype(np.float64))
        a = img1.detach().contiguous().float()
        b = img2.detach().contiguous().float()
        C = a.shape[2]
        out = torch.empty((ch, cw, C), dtype=torch.float32, device=img1.device)
        _lib.check(_lib.load().pysift_warp_f32_forward(a.data_ptr(), a.shape[0], a.shape[1], C, b.data_ptr(),
                                                       b.shape[0], b.shape[1], cw, ch,
                                                       hinv.ctypes.data_as(ctypes.c_void_p), ox, oy, iox, ioy,
                                                       out.data_ptr(), _st()), "pysift_warp_f32_forward")
        ctx.save_for_backward(a, b, Hinv)
        ctx.geometry = geometry
        ctx.hinv = hinv
        return out

    @staticmethod
    def backward(ctx, gout):
        a, b, Hinv = ctx.saved_tensors
        cw, ch, ox, oy, iox, ioy = ctx.geometry
        C = a.shape[2]
        g = gout.contiguous().float()
        ga = torch.zeros_like(a)
        gb = torch.zeros_like(b)
        gh = torch.zeros(9, dtype=torch.float64, device=a.device)
        _lib.check(_lib.load().pysift_warp_f32_backward(a.data_ptr(), a.shape[0], a.shape[1], C, b.data_ptr(),
                                                        b.shape[0], b.shape[1], cw, ch,
                                                        ctx.hinv.ctypes.data_as(ctypes.c_void_p), ox, oy, iox, ioy,
                                                        g.data_ptr(), ga.data_ptr(), gb.data_ptr(), gh.data_ptr(),
                                                        _st()), "pysift_warp_f32_backward")
        G = gh.reshape(3, 3)
        gH = -(Hinv.t() @ G @ Hinv.t())          # d(inv H) adjoint
        g8 = gH.reshape(-1)[:8]
        return ga, gb, g8, None


def warp_blend(img1, img2, h8, geometry):
    """Float warp + feather blend (ch, cw, C) of (H, W, C) float32 CUDA images;
    h8: the 8 homography parameters (row-major, H[2][2] = 1), view 1 -> view 2;
    geometry: canvas_geometry(...).  Differentiable in img1, img2 and h8."""
    return _WarpBlend.apply(img1, img2, h8, geometry)


def warp_blend_torch(img1, img2, h8, geometry):
    """warp_blend() restated with plain torch ops (autograd; any dtype)."""
    cw, ch, ox, oy, iox, ioy = geometry
    dt, dev = img1.dtype, img1.device
    Hinv = torch.linalg.inv(_h_from8(h8).to(dt))
    hs, ws, C = img1.shape
    h2, w2, _ = img2.shape
    v, u = torch.meshgrid(torch.arange(ch, device=dev, dtype=dt), torch.arange(cw, device=dev, dtype=dt),
                          indexing="ij")
    X, Y = u - ox, v - oy
    s0 = Hinv[0, 0] * X + Hinv[0, 1] * Y + Hinv[0, 2]
    s1 = Hinv[1, 0] * X + Hinv[1, 1] * Y + Hinv[1, 2]
    s2 = Hinv[2, 0] * X + Hinv[2, 1] * Y + Hinv[2, 2]
    den = torch.where(s2 >= 1e-10, s2, torch.full_like(s2, 1e-10))
    sx, sy = s0 / den, s1 / den
    v1 = (sx >= 0) & (sx <= ws - 1) & (sy >= 0) & (sy <= hs - 1)
    x0, y0 = torch.floor(sx).detach(), torch.floor(sy).detach()
    fx, fy = sx - x0, sy - y0

    def at(xx, yy):
        ok = (xx >= 0) & (xx < ws) & (yy >= 0) & (yy < hs)
        xi, yi = xx.clamp(0, ws - 1).long(), yy.clamp(0, hs - 1).long()
        return img1[yi, xi] * ok.unsqueeze(-1).to(dt)

    w1 = ((1 - fy) * (1 - fx)).unsqueeze(-1) * at(x0, y0) + ((1 - fy) * fx).unsqueeze(-1) * at(x0 + 1, y0) + \
         (fy * (1 - fx)).unsqueeze(-1) * at(x0, y0 + 1) + (fy * fx).unsqueeze(-1) * at(x0 + 1, y0 + 1)
    d1 = 1 + torch.minimum(torch.minimum(sx, ws - 1 - sx), torch.minimum(sy, hs - 1 - sy))
    ui, vi = torch.meshgrid(torch.arange(ch, device=dev), torch.arange(cw, device=dev), indexing="ij")
    x2, y2 = vi - iox, ui - ioy
    v2 = (x2 >= 0) & (x2 < w2) & (y2 >= 0) & (y2 < h2)
    i2 = img2[y2.clamp(0, h2 - 1), x2.clamp(0, w2 - 1)]
    d2 = (1 + torch.minimum(torch.minimum(x2, w2 - 1 - x2), torch.minimum(y2, h2 - 1 - y2))).to(dt)
    both = (v1 & v2).unsqueeze(-1)
    out = torch.where(both, (w1 * d1.unsqueeze(-1) + i2 * d2.unsqueeze(-1)) / (d1 + d2).unsqueeze(-1),
                      torch.where(v2.unsqueeze(-1), i2, torch.where(v1.unsqueeze(-1), w1, torch.zeros_like(w1))))
    return out
