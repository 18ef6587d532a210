"""detectAndCompute through the reference's own CUDA kernels -- TEST
INFRASTRUCTURE ONLY.

Drives the kernels oracle/build_ref.py compiles out of the reference's
pysift/core.py (oracle/_ref/libpysift_ref_kernels.so) with torch tensors on
the GPU, following the reference's host orchestration, PySIFT's B200 tier
(5 octaves unless given, float32 pyramid, 16 MP doubling cap):

  * contrast threshold: the value the product used is passed in (the
    reference's float32 CuPy entropy differs from it by rounding only);
  * base image gray / 255 in float32, the 2x cubic zoom by
    scipy.ndimage.zoom (the algorithm cupyx.scipy.ndimage.zoom implements;
    core.py:1270-1275), then gauss_h + gauss_v (_fast_gaussian,
    core.py:552-608) for the base blur and every level, next octave base =
    level S [::2, ::2] (core.py:1234-1352);
  * DoG in float32 (core.py:1354-1365); find_extrema_fused per octave; the
    candidates of each octave put in (s, r, c) order (the reference takes
    atomic-slot order; this harness canonicalises it, core.py:1367-1460);
    refine_keypoints (--use_fast_math) over all octaves' candidates;
  * starvation retry, 8000 cap by response (stable sort), core.py:2064-2080;
  * orientation_hist per octave, expansion in (keypoint, slot) order
    (core.py:1525-1603); sift_descriptor_coop per octave (core.py:1772-1858);
  * output order: stable lexsort by (x, y) (core.py:2111-2134).

Returns the rows before RootSIFT (the kernel's L2 / clip / L2 vector).
"""
import ctypes
import math
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libpysift_ref_kernels.so")
MAX_CANDS_PER_OCTAVE = 25000  # core.py:1395
BORDER = 5                    # core.py:1381

_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        vp, i32, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.ref_gaussian.argtypes = [vp, vp, vp, vp, i32, i32, i32, vp]
        L.ref_find_extrema.argtypes = [vp, vp, vp, i32, i32, i32, f32, i32, i32, vp]
        L.ref_refine.argtypes = [vp, vp, vp, i32, i32, i32, f32, f32, vp, vp, vp, vp, vp, vp, vp]
        L.ref_orientation.argtypes = [vp, vp, vp, i32, i32, i32, vp]
        L.ref_descriptor.argtypes = [vp, vp, vp, i32, i32, i32, i32, vp]
        _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: CUDA error {rc}")


def _weights(sigma, truncate=4):
    """core.py:572-577: numpy float32 weights."""
    radius = int(truncate * sigma + 0.5)
    x = np.arange(-radius, radius + 1, dtype=np.float32)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    return k.astype(np.float32), radius


class RefSIFT:
    def __init__(self, n_octaves=5, n_scales=3, sigma0=1.6, edge_thresh=10.0, double_image=True,
                 double_px_cap=16_000_000):
        import torch
        self.torch = torch
        self.n_octaves = n_octaves
        self.S = n_scales
        self.sigma0 = sigma0
        self.edge_thresh = edge_thresh
        self.double_image = double_image
        self.double_px_cap = double_px_cap
        self.dev = torch.device("cuda", 0)

    def _st(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def gaussian(self, img, sigma):
        """_fast_gaussian (core.py:552-608) with the reference's kernels."""
        torch = self.torch
        if sigma < 0.01:
            return img
        k, radius = _weights(sigma)
        kd = torch.from_numpy(k).to(self.dev)
        H, W = img.shape
        tmp = torch.empty((H, W), dtype=torch.float32, device=self.dev)
        out = torch.empty((H, W), dtype=torch.float32, device=self.dev)
        _check(lib().ref_gaussian(img.data_ptr(), tmp.data_ptr(), out.data_ptr(), kd.data_ptr(), H, W, radius,
                                  self._st()), "ref_gaussian")
        return out

    def pyramid(self, gray):
        torch = self.torch
        from scipy import ndimage
        S = self.S
        k = 2.0 ** (1.0 / S)
        sigmas = [self.sigma0 * (k ** s) for s in range(S + 3)]
        H, W = gray.shape
        base = (torch.from_numpy(gray).to(self.dev).to(torch.float32) / np.float32(255.0))
        self.doubled = bool(self.double_image and H * W < self.double_px_cap)
        if self.doubled:
            z = ndimage.zoom(base.cpu().numpy().astype(np.float32), 2.0, order=3)
            base = torch.from_numpy(np.ascontiguousarray(z, dtype=np.float32)).to(self.dev)
        assumed = 1.0 if self.doubled else 0.5
        sd0 = float(np.sqrt(max(self.sigma0 ** 2 - assumed ** 2, 1e-6)))
        inc = [float(np.sqrt(max(sigmas[s] ** 2 - sigmas[s - 1] ** 2, 1e-6))) for s in range(1, S + 3)]
        cur = self.gaussian(base.contiguous(), sd0)
        pyr = []
        for o in range(self.n_octaves):
            levels = [cur]
            prev = cur
            for s in range(S + 2):
                prev = self.gaussian(prev, inc[s])
                levels.append(prev)
            pyr.append(torch.stack(levels, 0).contiguous())
            cur = levels[S][::2, ::2].contiguous()
        return pyr

    def extrema_and_refine(self, dogs, ct):
        """_find_extrema + _refine_keypoints (core.py:1367-1523)."""
        torch = self.torch
        S = self.S
        thr = np.float32(ct / S)
        edge = np.float32((self.edge_thresh + 1.0) ** 2 / self.edge_thresh)
        cands, flat, meta, off = [], [], [], 0
        n_found = []
        for o, d in enumerate(dogs):
            S2, Ho, Wo = d.shape
            if Ho < 3 or Wo < 3:
                n_found.append(0)
                meta.append([S2, Ho, Wo, off])
                flat.append(d.reshape(-1))
                off += S2 * Ho * Wo
                continue
            coords = torch.empty(MAX_CANDS_PER_OCTAVE * 3, dtype=torch.int32, device=self.dev)
            count = torch.zeros(1, dtype=torch.int32, device=self.dev)
            _check(lib().ref_find_extrema(d.data_ptr(), coords.data_ptr(), count.data_ptr(), S2, Ho, Wo, float(thr),
                                          MAX_CANDS_PER_OCTAVE, BORDER, self._st()), "ref_find_extrema")
            n = int(count.item())
            n_found.append(n)
            n = min(n, MAX_CANDS_PER_OCTAVE)
            if n:
                c = coords[:3 * n].reshape(n, 3).cpu().numpy()
                c = c[np.lexsort((c[:, 2], c[:, 1], c[:, 0]))]  # canonical (s, r, c) order
                cands.append(np.column_stack([np.full(n, o, np.int32), c]).astype(np.int32))
            meta.append([S2, Ho, Wo, off])
            flat.append(d.reshape(-1))
            off += S2 * Ho * Wo
        if not cands:
            return [], n_found
        allc = np.ascontiguousarray(np.concatenate(cands))
        N = len(allc)
        dflat = torch.cat(flat).contiguous()
        dmeta = torch.from_numpy(np.array(meta, np.int32)).to(self.dev)
        dc = torch.from_numpy(allc).to(self.dev)
        outs = [torch.zeros(N, dtype=t, device=self.dev) for t in
                (torch.int32, torch.int32, torch.float32, torch.float32, torch.int32, torch.float32)]
        _check(lib().ref_refine(dflat.data_ptr(), dmeta.data_ptr(), dc.data_ptr(), N, S, BORDER, float(thr),
                                float(edge), *[t.data_ptr() for t in outs], self._st()), "ref_refine")
        valid, oct_, ri, ci, si, resp = [t.cpu().numpy() for t in outs]
        m = valid == 1
        refined = [(int(oct_[j]), int(si[j]), float(ri[j]), float(ci[j]), float(resp[j])) for j in np.nonzero(m)[0]]
        return refined, n_found

    def detect_and_compute(self, gray, ct):
        torch = self.torch
        S = self.S
        k_val = 2.0 ** (1.0 / S)
        pyr = self.pyramid(gray)
        dogs = [(g[1:] - g[:-1]).contiguous() for g in pyr]
        refined, n_found = self.extrema_and_refine(dogs, ct)
        retried = False
        if len(refined) < 100:
            refined, n_found = self.extrema_and_refine(dogs, ct * 0.5)
            retried = True
        if len(refined) > 8000:
            refined = sorted(refined, key=lambda t: t[4], reverse=True)[:8000]
        N = len(refined)
        res = dict(n_refined=N, n_cands=n_found, retried=retried, pyramid=pyr)
        if N == 0:
            return res
        oi = np.array([t[0] for t in refined], np.int32)
        si = np.array([t[1] for t in refined], np.float32)
        ri = np.array([t[2] for t in refined], np.float32)
        ci = np.array([t[3] for t in refined], np.float32)
        resp = np.array([t[4] for t in refined], np.float32)
        sigma = (self.sigma0 * (k_val ** si)).astype(np.float32)
        angles = np.full((N, 4), -1.0, np.float32)
        for o in np.unique(oi):
            m = np.nonzero(oi == o)[0]
            kp = torch.from_numpy(np.ascontiguousarray(np.column_stack([ri[m], ci[m], sigma[m], si[m]]),
                                                       np.float32)).to(self.dev)
            a = torch.empty((len(m), 4), dtype=torch.float32, device=self.dev)
            g = pyr[o]
            _check(lib().ref_orientation(g.data_ptr(), kp.data_ptr(), a.data_ptr(), len(m), g.shape[1], g.shape[2],
                                         self._st()), "ref_orientation")
            angles[m] = a.cpu().numpy()
        vi, vj = np.nonzero(angles >= 0.0)
        ang = angles[vi, vj]
        o2, si2, ri2, ci2, resp2 = oi[vi], si[vi], ri[vi], ci[vi], resp[vi]
        ang_rad = np.radians(ang)
        ph = np.maximum(4.0, np.round(3.0 * self.sigma0 * (k_val ** si2) * math.sqrt(2) * 2.5)).astype(np.float32)
        desc = np.zeros((len(vi), 128), np.float32)
        for o in np.unique(o2):
            m = np.nonzero(o2 == o)[0]
            kp = torch.from_numpy(np.ascontiguousarray(np.column_stack([ri2[m], ci2[m], ang_rad[m], ph[m], si2[m]]),
                                                       np.float32)).to(self.dev)
            d = torch.empty((len(m), 128), dtype=torch.float32, device=self.dev)
            g = pyr[o]
            _check(lib().ref_descriptor(g.data_ptr(), kp.data_ptr(), d.data_ptr(), len(m), g.shape[0], g.shape[1],
                                        g.shape[2], self._st()), "ref_descriptor")
            desc[m] = d.cpu().numpy()
        cs = 0.5 if self.doubled else 1.0
        xs = np.array([float(c) * float(2 ** int(o)) * cs for c, o in zip(ci2, o2)], np.float32)
        ys = np.array([float(r) * float(2 ** int(o)) * cs for r, o in zip(ri2, o2)], np.float32)
        sz = np.array([self.sigma0 * (k_val ** int(s)) * float(2 ** int(o)) * cs * 2.0 for s, o in zip(si2, o2)],
                      np.float32)
        order = np.lexsort((ys, xs))
        res.update(x=xs[order], y=ys[order], size=sz[order], angle=ang[order], response=resp2[order],
                   octave=o2[order].astype(np.int32), desc=desc[order])
        return res
