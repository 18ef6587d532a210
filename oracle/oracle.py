"""CPU oracle for the PySIFT hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product (pysift_b200) never does.  It restates the
reference's host orchestration in numpy and calls the C restatement of its
kernels (oracle/sift_oracle.c, built by oracle/build_oracle.sh).

Reference: pysift/core.py of SivaIITM/PySIFT (staysift 0.1.4).  Canonical
choices where the reference is order-dependent or approximate are listed in
sift_oracle.c's header; the orchestration-level ones are:
  * candidates are taken per octave in (s, r, c) order (the reference uses
    atomic-slot order), so refined keypoints are in (octave, s, r, c) order;
  * the entropy threshold is computed in float64 (reference: CuPy float32).
"""
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.check_call([os.path.join(_HERE, "build_oracle.sh")])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_contrast_thresh.restype = ctypes.c_double
        _lib.orc_contrast_thresh.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double]
        _lib.orc_find_extrema.restype = ctypes.c_long
        _lib.orc_find_extrema.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _lib.orc_refine.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_float, ctypes.c_float] + [ctypes.c_void_p] * 5
        _lib.orc_gauss_blur.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_int]
        _lib.orc_zoom2x.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _lib.orc_orientation.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_long, ctypes.c_void_p]
        _lib.orc_descriptor.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p]
        _lib.orc_rootsift.argtypes = [ctypes.c_void_p, ctypes.c_long]
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


MAX_CANDS_PER_OCTAVE = 25000   # pysift/core.py:1395
BORDER = 5                      # pysift/core.py:1381
KEYPOINT_CAP = 8000             # pysift/core.py:2078
STARVATION_MIN = 100            # pysift/core.py:2066

DSP_PRESETS = {                 # pysift/core.py:1198-1202
    3: np.array([1.0 / math.sqrt(2), 1.0, math.sqrt(2)], dtype=np.float32),
    4: np.array([0.5, 1.0 / math.sqrt(2), 1.0, math.sqrt(2)], dtype=np.float32),
    5: np.array([0.5, 1.0 / math.sqrt(2), 1.0, math.sqrt(2), 2.0], dtype=np.float32),
}


def gaussian_weights(sigma, truncate=4):
    """1-D weights as pysift/core.py:563-577 builds them (numpy float32)."""
    radius = int(truncate * sigma + 0.5)
    x = np.arange(-radius, radius + 1, dtype=np.float32)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    return k.astype(np.float32), radius


def gauss_blur(img, sigma, truncate=4):
    """_fast_gaussian (pysift/core.py:552-608)."""
    if sigma < 0.01:
        return img
    k, radius = gaussian_weights(sigma, truncate)
    H, W = img.shape
    src = np.ascontiguousarray(img, dtype=np.float32)
    out = np.empty((H, W), np.float32)
    lib().orc_gauss_blur(_p(src), _p(out), H, W, _p(k), radius)
    return out


def contrast_thresh(gray, base=0.04):
    g = np.ascontiguousarray(gray, dtype=np.uint8)
    return lib().orc_contrast_thresh(_p(g), g.size, base)


def zoom2x(img):
    H, W = img.shape
    src = np.ascontiguousarray(img, dtype=np.float32)
    out = np.empty((2 * H, 2 * W), np.float32)
    lib().orc_zoom2x(_p(src), H, W, _p(out))
    return out


class OracleSIFT:
    """Restatement of PySIFT (pysift/core.py:1150-2172) on the CPU."""

    def __init__(self, n_octaves=None, n_scales=3, sigma0=1.6, contrast_thresh=0.04,
                 edge_thresh=10.0, dsp=False, dsp_n_scales=3, fp16_pyramid=None,
                 double_image=True, rootsift=True, high_vram=True):
        self.high_vram = high_vram
        self.n_octaves = n_octaves if n_octaves is not None else (5 if high_vram else 4)
        self.n_scales = n_scales
        self.sigma0 = sigma0
        self.contrast_thresh = contrast_thresh
        self.edge_thresh = edge_thresh
        self.dsp = dsp
        self.dsp_scales = DSP_PRESETS[dsp_n_scales]
        self.fp16_pyramid = fp16_pyramid if fp16_pyramid is not None else (not high_vram)
        self.double_image = double_image
        self.rootsift = rootsift

    # pysift/core.py:1234-1352
    def build_pyramid(self, gray):
        S = self.n_scales
        k = 2.0 ** (1.0 / S)
        sigmas = [self.sigma0 * (k ** s) for s in range(S + 3)]
        H, W = gray.shape
        base = gray.astype(np.float32) / np.float32(255.0)
        if self.fp16_pyramid:
            base = base.astype(np.float16).astype(np.float32)
        cap = 16_000_000 if self.high_vram else 4_194_304
        self.effective_double = bool(self.double_image and (H * W < cap))
        if self.effective_double:
            base = zoom2x(base)
            if self.fp16_pyramid:
                base = base.astype(np.float16).astype(np.float32)
        assumed_blur = 1.0 if self.effective_double else 0.5
        sd0 = float(np.sqrt(max(self.sigma0 ** 2 - assumed_blur ** 2, 1e-6)))
        inc = [float(np.sqrt(max(sigmas[s] ** 2 - sigmas[s - 1] ** 2, 1e-6))) for s in range(1, S + 3)]
        cur = gauss_blur(base, sd0)
        pyr = []
        for o in range(self.n_octaves):
            levels = [cur]
            prev = cur
            for s in range(S + 2):
                prev = gauss_blur(prev, inc[s])
                levels.append(prev)
            stack = np.stack(levels, 0)
            if self.fp16_pyramid and o >= 2:
                stack = stack.astype(np.float16).astype(np.float32)
            pyr.append(stack)
            cur = np.ascontiguousarray(levels[S][::2, ::2])
        return pyr

    @staticmethod
    def dog(pyr):
        return [np.ascontiguousarray(g[1:] - g[:-1]) for g in pyr]

    # pysift/core.py:1367-1523
    def extrema_and_refine(self, dogs, ct):
        S = self.n_scales
        thr = np.float32(ct / S)
        edge = np.float32((self.edge_thresh + 1.0) ** 2 / self.edge_thresh)
        out = []
        n_cands = []
        for o, d in enumerate(dogs):
            S2, H, W = d.shape
            if H < 3 or W < 3:
                n_cands.append(0)
                continue
            coords = np.empty((MAX_CANDS_PER_OCTAVE, 3), np.int32)
            found = lib().orc_find_extrema(_p(d), S2, H, W, float(thr), BORDER, MAX_CANDS_PER_OCTAVE, _p(coords))
            n = min(found, MAX_CANDS_PER_OCTAVE)
            n_cands.append(int(found))
            if n == 0:
                continue
            c = np.ascontiguousarray(coords[:n])
            valid = np.zeros(n, np.int32)
            ri = np.zeros(n, np.float32)
            ci = np.zeros(n, np.float32)
            si = np.zeros(n, np.int32)
            resp = np.zeros(n, np.float32)
            lib().orc_refine(_p(d), S2, H, W, _p(c), n, S, BORDER, float(thr), float(edge),
                             _p(valid), _p(ri), _p(ci), _p(si), _p(resp))
            m = valid == 1
            for j in np.nonzero(m)[0]:
                out.append((o, int(si[j]), float(ri[j]), float(ci[j]), float(resp[j]),
                            tuple(int(v) for v in c[j])))
        return out, n_cands

    def detect_and_compute(self, gray):
        """Returns a dict with the reference's outputs in its final order."""
        S = self.n_scales
        k_val = 2.0 ** (1.0 / S)
        ct = contrast_thresh(gray, self.contrast_thresh)
        pyr = self.build_pyramid(gray)
        dogs = self.dog(pyr)
        refined, n_cands = self.extrema_and_refine(dogs, ct)
        retried = False
        if len(refined) < STARVATION_MIN:
            refined, n_cands = self.extrema_and_refine(dogs, ct * 0.5)
            retried = True
        capped = False
        if len(refined) > KEYPOINT_CAP:
            refined = sorted(refined, key=lambda t: t[4], reverse=True)[:KEYPOINT_CAP]
            capped = True
        N = len(refined)
        info = dict(ct=ct, n_cands=n_cands, n_refined=N, retried=retried, capped=capped,
                    effective_double=self.effective_double, pyramid=pyr)
        if N == 0:
            info.update(x=np.zeros(0, np.float32), y=np.zeros(0, np.float32),
                        size=np.zeros(0, np.float32), angle=np.zeros(0, np.float32),
                        response=np.zeros(0, np.float32), octave=np.zeros(0, np.int32),
                        desc=np.zeros((0, 128), np.float32))
            return info
        oi = np.array([t[0] for t in refined], np.int32)
        si_f = np.array([t[1] for t in refined], np.float32)
        ri = np.array([t[2] for t in refined], np.float32)
        ci = np.array([t[3] for t in refined], np.float32)
        resp = np.array([t[4] for t in refined], np.float32)
        # orientation (pysift/core.py:1525-1603)
        sigma = (self.sigma0 * (k_val ** si_f)).astype(np.float32)
        angles = np.full((N, 4), -1.0, np.float32)
        for o in np.unique(oi):
            m = np.nonzero(oi == o)[0]
            kp = np.ascontiguousarray(np.column_stack([ri[m], ci[m], sigma[m], si_f[m]]).astype(np.float32))
            g = pyr[o]
            a = np.empty((len(m), 4), np.float32)
            lib().orc_orientation(_p(g), g.shape[1], g.shape[2], _p(kp), len(m), _p(a))
            angles[m] = a
        vi, vj = np.nonzero(angles >= 0.0)
        n2 = len(vi)
        ang = angles[vi, vj]
        o2, si2, ri2, ci2, resp2 = oi[vi], si_f[vi], ri[vi], ci[vi], resp[vi]
        # descriptor (pysift/core.py:1772-1900)
        ang_rad = np.radians(ang)
        ph = np.maximum(4.0, np.round(3.0 * self.sigma0 * (k_val ** si2) * math.sqrt(2) * 2.5)).astype(np.float32)
        desc = np.zeros((n2, 128), np.float32)
        for o in np.unique(o2):
            m = np.nonzero(o2 == o)[0]
            kp = np.ascontiguousarray(np.column_stack([ri2[m], ci2[m], ang_rad[m], ph[m], si2[m]]).astype(np.float32))
            g = pyr[o]
            d = np.empty((len(m), 128), np.float32)
            if self.dsp:
                sc = np.ascontiguousarray(self.dsp_scales)
                lib().orc_descriptor(_p(g), g.shape[0], g.shape[1], g.shape[2], _p(kp), len(m), _p(sc), len(sc), _p(d))
            else:
                lib().orc_descriptor(_p(g), g.shape[0], g.shape[1], g.shape[2], _p(kp), len(m), None, 0, _p(d))
            desc[m] = d
        info["desc_l2"] = desc.copy()
        if self.rootsift:
            lib().orc_rootsift(_p(desc), n2)
        # output assembly (pysift/core.py:1491-1522, 2111-2142)
        cs = 0.5 if self.effective_double else 1.0
        xs = np.array([float(c) * float(2 ** int(o)) * cs for c, o in zip(ci2, o2)], np.float32)
        ys = np.array([float(r) * float(2 ** int(o)) * cs for r, o in zip(ri2, o2)], np.float32)
        sz = np.array([self.sigma0 * (k_val ** int(s)) * float(2 ** int(o)) * cs * 2.0
                       for s, o in zip(si2, o2)], np.float32)
        order = np.lexsort((ys, xs))
        info.update(x=xs[order], y=ys[order], size=sz[order], angle=ang[order], response=resp2[order],
                    octave=o2[order].astype(np.int32), desc=desc[order], desc_l2=info["desc_l2"][order])
        return info
