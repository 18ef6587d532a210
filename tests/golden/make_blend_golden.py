"""Regenerates tests/golden/blend_cases.npz: the reference's own composition
(GPUPyStitch._blend_pair -- gain, _find_seam with the DP seams and the
sigma-3 mask blur, _multiband_blend -- and the paste of _stitch_pair) run on
small synthetic canvases, and tests/golden/triple_cases.npz: the
reference's _stitch_triple on three small synthetic views, its stages before
the composition (preprocessing, features, matching, RANSAC, depth) replaced
by stubs that hand it fixed homographies, so that its own warps, two-pass
composition, paste and inner-rectangle crop run unchanged.

pysift/core.py imports cupy, cupyx.scipy.ndimage and numba at module level
and this machine has no GPU, so the script puts numpy in place of cupy and
scipy.ndimage in place of cupyx.scipy.ndimage (the module cupyx mirrors);
numba's decorators become no-ops (none of the numba kernels is on this path).
Everything else is the reference's code as it lies in its tree.

    python tests/golden/make_blend_golden.py /path/to/reference [output_dir]
"""
import os
import sys
import types

import numpy as np
import scipy.ndimage

HERE = os.path.dirname(os.path.abspath(__file__))


class _Anything:
    """Stands in for numba: every attribute and call yields itself, and a
    decorator applied to a function returns the function."""

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Anything()

    def __call__(self, *a, **k):
        if len(a) == 1 and callable(a[0]) and not k:
            return a[0]
        return _Anything()


def _module_getattr(get):
    def __getattr__(name):
        if name.startswith("__"):
            raise AttributeError(name)
        return get(name)
    return __getattr__


def _install_shims():
    cp = types.ModuleType("cupy")
    # numpy where it has the name; module-level kernels (cp.fuse, RawKernel)
    # that this path never calls become placeholders
    cp.__getattr__ = _module_getattr(lambda name: getattr(np, name) if hasattr(np, name) else _Anything())

    class _Pool:
        def free_all_blocks(self):
            pass

    cp.asarray = np.asarray
    cp.asnumpy = np.asarray
    cp._default_memory_pool = _Pool()
    cp.get_default_memory_pool = lambda: _Pool()
    cupyx = types.ModuleType("cupyx")
    cupyx_scipy = types.ModuleType("cupyx.scipy")
    cupyx.scipy = cupyx_scipy
    cupyx_scipy.ndimage = scipy.ndimage
    sys.modules.update({"cupy": cp, "cupyx": cupyx, "cupyx.scipy": cupyx_scipy,
                        "cupyx.scipy.ndimage": scipy.ndimage})
    nb = types.ModuleType("numba")
    nb.__getattr__ = _module_getattr(lambda name: _Anything())
    nb.cuda = _Anything()
    sys.modules["numba"] = nb
    sys.modules["numba.cuda"] = nb.cuda


def _texture(rng, h, w, scale):
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    base = 110 + 60 * np.sin(x / 9.0 + 0.5) * np.cos(y / 13.0) + 25 * np.sin((x + 2 * y) / 5.0)
    img = np.stack([base * s for s in scale], axis=2) + rng.normal(0, 6, (h, w, 3))
    return np.clip(img, 0, 255).astype(np.uint8)


def make_cases():
    """(name, warped1, mask1, canvas2, mask2) for the seam orientations, the
    side of image 1, gain clipping and the no-overlap case."""
    rng = np.random.default_rng(20240611)
    cases = []
    ch, cw = 72, 150
    yy, xx = np.mgrid[0:ch, 0:cw]
    # vertical seam, image 1 on the left (a slanted right edge)
    m1 = (xx < 96 + (yy * 0.25).astype(int)) & (yy > 2 + xx // 30)
    m2 = (xx >= 58) & (yy >= 4) & (yy < 70)
    w1 = _texture(rng, ch, cw, (1.0, 0.9, 0.8))
    w1[~m1] = (rng.random((int((~m1).sum()), 3)) < 0.05) * 37  # stray values off the mask
    c2 = _texture(rng, ch, cw, (0.95, 1.0, 0.85))
    c2[~m2] = 0
    cases.append(("vertical_left", w1, m1, c2, m2))
    # vertical seam, image 1 on the right
    cases.append(("vertical_right", w1[:, ::-1].copy(), m1[:, ::-1].copy(), c2[:, ::-1].copy(),
                  m2[:, ::-1].copy()))
    # horizontal seam (stacked views), image 1 below; image 1 dark enough to clip the gain at 2
    ch2, cw2 = 128, 96
    yy, xx = np.mgrid[0:ch2, 0:cw2]
    m1 = (yy >= 50 - xx // 12) & (xx > 3)
    m2 = (yy < 84) & (xx < 90)
    w1 = (_texture(rng, ch2, cw2, (0.4, 0.45, 0.35))).astype(np.uint8)
    w1[~m1] = 0
    c2 = _texture(rng, ch2, cw2, (1.0, 1.0, 1.0))
    c2[~m2] = 0
    cases.append(("horizontal_below_gainclip", w1, m1, c2, m2))
    # no overlap
    ch3, cw3 = 40, 90
    yy, xx = np.mgrid[0:ch3, 0:cw3]
    m1 = xx < 40
    m2 = xx >= 45
    w1 = _texture(rng, ch3, cw3, (1.0, 1.0, 1.0))
    w1[~m1] = 0
    c2 = _texture(rng, ch3, cw3, (0.9, 0.9, 0.9))
    c2[~m2] = 0
    cases.append(("no_overlap", w1, m1, c2, m2))
    return cases


def make_triples():
    """(name, img1, img2, img3, H12, H32): views of one texture, image 1 left
    of image 2 and image 3 right of it, with a little rotation / perspective."""
    rng = np.random.default_rng(77)
    out = []
    for k, (h, w, sh1, sh3) in enumerate([(90, 120, 70, 74), (72, 100, 58, 61)]):
        big = _texture(rng, h + 20, 3 * w, (1.0, 0.92, 0.85))
        c2 = w  # image 2 starts here; image 1 sh1 columns left of it, image 3 sh3 right
        img1 = big[10:10 + h, c2 - sh1:c2 - sh1 + w].copy()
        img2 = big[10:10 + h, c2:c2 + w].copy()
        img3 = big[10:10 + h, c2 + sh3:c2 + sh3 + w].copy()
        img3 = np.clip(img3.astype(np.float32) * np.float32(0.9) + 6, 0, 255).astype(np.uint8)
        a = 0.01 * (k + 1)
        H12 = np.array([[np.cos(a), -np.sin(a), -float(sh1)], [np.sin(a), np.cos(a), 1.5], [2e-5, 0, 1.0]])
        H32 = np.array([[1.0, 0.0, float(sh3)], [0.0, 1.0, -1.0], [0.0, -1e-5, 1.0]])
        out.append((f"triple{k}", img1, img2, img3, H12, H32))
    return out


def run_triples(st_cls, out_dir):
    import cv2
    res = {}
    names = []
    for name, img1, img2, img3, H12, H32 in make_triples():
        st = object.__new__(st_cls)
        st.color_match = "gain"
        st.n_blend_levels = 6
        st.n_depth_layers = 4
        kps = [cv2.KeyPoint(float(i), float(i), 1.0) for i in range(12)]
        dms = [cv2.DMatch(i, i, 0.0) for i in range(12)]
        hs = iter([H12, H32])
        st._preprocess_image = lambda img: img
        st._extract_features = lambda img: (kps, None, None)
        st._match_features = lambda *a: dms
        st._compute_homography = lambda *a: None
        st._ransac = lambda p, q: (next(hs), np.ones(len(p), bool))
        st._get_depth_estimator = lambda: None
        warps = []
        orig = st_cls._warp_image

        def rec(img, H, cw, ch, ox, oy, _orig=orig):
            w, m = _orig(img, H, cw, ch, ox, oy)
            warps.append((w, m))
            return w, m

        st._warp_image = rec
        pano, _, metrics = st._stitch_triple(img1, img2, img3)
        cw, ch, ox, oy = st_cls._compute_canvas_size_3(img1, img2, img3, H12, H32)
        iox, ioy = int(round(ox)), int(round(oy))
        canvas2 = np.zeros((ch, cw, 3), np.uint8)
        mask2 = np.zeros((ch, cw), bool)
        ye, xe = min(ioy + img2.shape[0], ch), min(iox + img2.shape[1], cw)
        canvas2[ioy:ye, iox:xe] = img2[:ye - ioy, :xe - iox]
        mask2[ioy:ye, iox:xe] = True
        names.append(name)
        res.update({f"{name}_img1": img1, f"{name}_img2": img2, f"{name}_img3": img3, f"{name}_H12": H12,
                    f"{name}_H32": H32, f"{name}_warped1": warps[0][0], f"{name}_mask1": warps[0][1],
                    f"{name}_warped3": warps[1][0], f"{name}_mask3": warps[1][1], f"{name}_canvas2": canvas2,
                    f"{name}_mask2": mask2, f"{name}_pano": pano,
                    f"{name}_seam_rmse": np.float64(metrics["seam_rmse"]),
                    f"{name}_seam_rmse_23": np.float64(metrics["seam_rmse_23"])})
        print(name, "canvas", (cw, ch), "pano", pano.shape, "rmse", metrics["seam_rmse"], metrics["seam_rmse_23"])
    res["names"] = np.array(names)
    np.savez_compressed(os.path.join(out_dir, "triple_cases.npz"), **res)


def main(ref_root, out_dir=HERE):
    sys.dont_write_bytecode = True
    _install_shims()
    sys.path.insert(0, ref_root)
    from pysift.core import GPUPyStitch
    st = object.__new__(GPUPyStitch)
    st.color_match = "gain"
    st.n_blend_levels = 6
    out = {}
    names = []
    for name, w1, m1, c2, m2 in make_cases():
        ch, cw = m1.shape
        blended, both, rmse = st._blend_pair(w1.astype(np.float32), m1, c2.astype(np.float32), m2, cw, ch)
        pano = np.zeros((ch, cw, 3), np.uint8)
        pano[both] = np.clip(blended[both], 0, 255).astype(np.uint8)
        names.append(name)
        out.update({f"{name}_warped1": w1, f"{name}_mask1": m1, f"{name}_canvas2": c2, f"{name}_mask2": m2,
                    f"{name}_pano": pano, f"{name}_both": both, f"{name}_seam_rmse": np.float64(rmse)})
        print(name, pano.shape, "rmse", rmse)
        # the same canvases with histogram matching in place of the gain (core.py:3694-3695)
        st.color_match = "hist"
        blended, both, rmse = st._blend_pair(w1.astype(np.float32), m1, c2.astype(np.float32), m2, cw, ch)
        st.color_match = "gain"
        pano = np.zeros((ch, cw, 3), np.uint8)
        pano[both] = np.clip(blended[both], 0, 255).astype(np.uint8)
        out.update({f"{name}_hist_pano": pano, f"{name}_hist_seam_rmse": np.float64(rmse)})
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(out_dir, "blend_cases.npz"), **out)
    run_triples(GPUPyStitch, out_dir)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else ".", sys.argv[2] if len(sys.argv) > 2 else HERE)
