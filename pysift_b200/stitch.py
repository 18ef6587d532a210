"""GPUPyStitch drop-in (pysift/core.py:2401-4092) on the B200 kernels.

The two-image path of the reference -- BGR->gray, CLAHE, SIFT, top-k by
response, L2 + PCA-64 + fp16 mutual ratio-test matching, batched RANSAC with
MAGSAC++ scoring and LO refits, canvas, bilinear warp -- runs as C-ABI calls
on the current CUDA stream.  Composition (blend='multiband', the default) is
the reference's: gain compensation, dynamic-programming seam and a 6-level
Laplacian blend (pysift/core.py:3386-3553, 3686-3714) on the device;
blend='feather' swaps in a linear feather blend (weights 1 + distance to
each image's border).  Both end with the reference's inner-rectangle crop.
The host reads back only the homography (72 bytes + 3 counters) to size the
canvas, the coverage extents for the crop and the final panorama.
"""
import ctypes
import os
import time
from datetime import datetime

import numpy as np
import torch

from . import _lib
from .core import PySIFT, capture_graph, check_detector_options

#: host threads of the staging copy of a host image (pysift_host_copy), used
#: from _STAGE_THREADED_BYTES up.  On a B200 host the 4-thread copy of a
#: 3.7 MB view takes 0.04 ms against 0.20 ms for one thread, yet the
#: end-to-end stitch of a 1280x960 pair was slower with it (3.46 against
#: 3.25 ms median); the 32-pair batch of views up to 3000x2000 (18 MB) went
#: from 151 to 223 pairs/s end to end with it.
_STAGE_THREADS = max(1, min(4, os.cpu_count() or 1))
_STAGE_THREADED_BYTES = 8 << 20


def _ptr_aligned(t, align=256):
    off = (-t.data_ptr()) % align
    return t.data_ptr() + off, t.numel() * t.element_size() - off


class _Dev:
    """Per-size device scratch reused across calls."""

    def __init__(self):
        self.bufs = {}

    def get(self, key, shape, dtype, device):
        t = self.bufs.get(key)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=device)
            self.bufs[key] = t
        return t


class GPUPyStitch:
    """Panorama stitcher with the reference's constructor (pysift/core.py:2429-2445).

    Not thread-safe (per-instance buffers and the cached PCA basis, like the
    reference).  Two and three images are supported; depth-aware warps,
    learned features and LightGlue raise NotImplementedError.
    """

    def __init__(self, n_depth_layers=4, n_blend_levels=6, ransac_iters=1500, inlier_thresh=5.0,
                 ransac_method='magsac', sigma_max=None, match_ratio=0.75, match_batch=512, max_keypoints=8000,
                 pca_dims=64, int8_matching=False, orientation='histogram', descriptor='sift', matcher='ratio',
                 color_match='gain', dsp_sift=False, contrast_thresh=0.04, n_octaves=4, n_scales=3, sigma0=1.6,
                 edge_thresh=10.0, double_image=True, max_dimension=0, denoise=False, sharpen=False,
                 clahe_clip=2.0, clahe_tile=8, output_max_dim=0, post_sharpen=False, output_format='png',
                 output_quality=90, *, device=None, save_output=True, verbose=True, high_vram=None,
                 blend='multiband'):
        check_detector_options(3, orientation, descriptor)
        if matcher != 'ratio':
            raise NotImplementedError(f"matcher={matcher!r}: only the ratio-test matcher is implemented here")
        if pca_dims not in (0, 64, 128):
            raise NotImplementedError("pca_dims must be 0, 64 or 128 on this backend")
        if blend not in ('multiband', 'feather'):
            raise ValueError(f"blend must be 'multiband' or 'feather' (got {blend!r})")
        if blend == 'multiband' and not 1 <= int(n_blend_levels) <= 8:
            raise ValueError("n_blend_levels must be within 1..8")
        if ransac_method not in ('magsac', 'classic'):
            raise ValueError(f"ransac_method must be 'magsac' or 'classic' (got {ransac_method!r})")
        self.n_depth_layers = n_depth_layers
        self.n_blend_levels = n_blend_levels
        self.blend = blend
        self.ransac_iters = ransac_iters
        self.inlier_thresh = inlier_thresh
        self.ransac_method = ransac_method
        self.sigma_max = sigma_max if sigma_max is not None else inlier_thresh
        self.match_ratio = match_ratio
        self.match_batch = match_batch
        self.max_keypoints = max_keypoints
        self.pca_dims = pca_dims
        self.int8_matching = int8_matching
        self.matcher = matcher
        self.descriptor = descriptor
        self.color_match = color_match
        self.max_dimension = max_dimension
        self.denoise = denoise
        self.sharpen = sharpen
        self.clahe_clip = clahe_clip
        self.clahe_tile = clahe_tile
        self.output_max_dim = output_max_dim
        self.post_sharpen = post_sharpen
        self.output_format = output_format.lower()
        self.output_quality = output_quality
        self.save_output = save_output
        self.verbose = verbose
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._detector = PySIFT(dsp=dsp_sift, orientation=orientation, descriptor=descriptor, n_octaves=n_octaves,
                                n_scales=n_scales, sigma0=sigma0, contrast_thresh=contrast_thresh,
                                edge_thresh=edge_thresh, double_image=double_image, device=self.device,
                                high_vram=high_vram)
        # the detector describes only the top max_keypoints by response, in
        # the order of the reference's stable selection (pysift/core.py:2566-2571)
        self._detector._cfg.output_limit = int(max_keypoints)
        self._lib = _lib.load()
        self._dev = _Dev()
        self._pca_matrix = None   # float32 (128, pca_dims) on the device, fitted on the first pair
        self._pca_mean = None
        self._rand = {}
        self.last_metrics = None
        self.last_timings = None
        self.stage_events = None  # optional list of 6 torch.cuda.Event(enable_timing=True)
        self._side = None         # two side streams, one per view
        self._graphs = {}         # captured match + RANSAC launches per (counts, buffers)

    # ------------------------------------------------------------------
    #: stage names of the events recorded when ``stage_events`` holds six
    #: CUDA events: upload + CLAHE + detection of both views (concurrent),
    #: top-k + matcher preparation, matching, RANSAC, warp + blend + crop
    STAGES = ("features", "prep", "match", "ransac", "compose")

    def _mark(self, i):
        ev = getattr(self, "stage_events", None)
        if ev is not None:
            ev[i].record(torch.cuda.current_stream(self.device))

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _upload_bgr(self, img, key):
        if isinstance(img, torch.Tensor) and img.is_cuda:
            return img.contiguous()
        img = np.ascontiguousarray(img)
        if img.dtype != np.uint8 or img.ndim != 3 or img.shape[2] != 3:
            raise ValueError("images must be BGR uint8 arrays of shape (H, W, 3)")
        host = self._dev.bufs.get(key + "_host")
        if host is None or tuple(host.shape) != img.shape:
            host = torch.empty(img.shape, dtype=torch.uint8).pin_memory()
            self._dev.bufs[key + "_host"] = host
        # staging copy, on several host threads for large images (the GIL is
        # released in the call)
        threads = _STAGE_THREADS if img.nbytes >= _STAGE_THREADED_BYTES else 1
        _lib.check(self._lib.pysift_host_copy(host.data_ptr(), img.ctypes.data, img.nbytes, threads),
                   "pysift_host_copy")
        dev = self._dev.get(key, img.shape, torch.uint8, self.device)
        dev.copy_(host, non_blocking=True)
        return dev

    def _gray_clahe(self, bgr, key):
        """BGR -> gray -> CLAHE on the device (pysift/core.py:2545-2565)."""
        H, W = bgr.shape[:2]
        st = self._stream()
        gray = self._dev.get(key + "_gray", (H, W), torch.uint8, self.device)
        _lib.check(self._lib.pysift_bgr2gray(bgr.data_ptr(), H, W, bgr.stride(0), gray.data_ptr(), W, st),
                   "pysift_bgr2gray")
        if self.clahe_clip is None:
            return gray
        t = int(self.clahe_tile)
        lut = self._dev.get(key + "_lut", (t * t * 256,), torch.uint8, self.device)
        out = self._dev.get(key + "_clahe", (H, W), torch.uint8, self.device)
        _lib.check(self._lib.pysift_clahe(gray.data_ptr(), H, W, W, float(self.clahe_clip), t, t, lut.data_ptr(),
                                          out.data_ptr(), W, st), "pysift_clahe")
        return out

    def _detect_view(self, img, key, slot, stream):
        """Upload (host images), gray + CLAHE and detection of one view,
        enqueued on `stream`; the keypoint count is copied to pinned host
        memory on the same stream."""
        with torch.cuda.stream(stream):
            bgr = self._upload_bgr(img, key)
            g = self._gray_clahe(bgr, key)
            b = self._detector.run_device(g, slot=slot)
            b.stats_host.copy_(b.stats, non_blocking=True)
        return bgr, b

    def _select(self, b, key):
        """Keypoints and descriptors of one view: the detector already kept the
        top max_keypoints by response (stable, pysift/core.py:2566-2571).
        Returns device views (kpts (N,4), desc (N,128), N); the stats must be
        on the host."""
        n = int(b.stats_host[_lib.STAT_N_KEYPOINTS])
        return b.kpts[:n], b.desc[:n], n

    def _features(self, bgr, key):
        """Detect + describe one view on the current stream, then select."""
        st = torch.cuda.current_stream(self.device)
        _, b = self._detect_view(bgr, key, 0, st)
        st.synchronize()
        return self._select(b, key)

    def _prepare(self, d1, d2):
        """L2-normalise, PCA (fitted once per instance), then fp16 or, with
        int8_matching, per-row int8 quantisation (pysift/core.py:2877-2905).
        Returns ("f16", a, b) or ("i8", q1, s1, q2, s2) for _match_prepared."""
        st = self._stream()
        lib = self._lib
        n1, n2 = d1.shape[0], d2.shape[0]
        D = d1.shape[1]
        both = torch.empty((n1 + n2, D), dtype=torch.float32, device=self.device)
        _lib.check(lib.pysift_l2_normalize_rows(d1.data_ptr(), n1, D, both.data_ptr(), st), "l2")
        _lib.check(lib.pysift_l2_normalize_rows(d2.data_ptr(), n2, D, both[n1:].data_ptr(), st), "l2")
        P = self.pca_dims if (self.descriptor == 'sift' and 0 < self.pca_dims < D) else 0
        if P == 0:
            if self.int8_matching:
                return self._quantize(both[:n1], both[n1:])
            out = torch.empty((n1 + n2, D), dtype=torch.float16, device=self.device)
            _lib.check(lib.pysift_to_f16(both.data_ptr(), both.numel(), out.data_ptr(), st), "to_f16")
            return ("f16", out[:n1], out[n1:])
        if self._pca_matrix is None:
            mean = torch.empty(D, dtype=torch.float32, device=self.device)
            cov = torch.empty((D, D), dtype=torch.float64, device=self.device)
            sz = ctypes.c_size_t()
            _lib.check(lib.pysift_pca_workspace_size(n1 + n2, D, ctypes.byref(sz)), "pysift_pca_workspace_size")
            ws = torch.empty(int(sz.value), dtype=torch.uint8, device=self.device)
            _lib.check(lib.pysift_pca_stats(both.data_ptr(), n1 + n2, D, ws.data_ptr(), ws.numel(), mean.data_ptr(),
                                            cov.data_ptr(), st), "pysift_pca_stats")
            # one 128x128 symmetric eigendecomposition per instance (parallel
            # Jacobi on the device), the basis cached like the reference's
            # (pysift/core.py:2729-2736)
            proj = torch.empty((D, P), dtype=torch.float32, device=self.device)
            _lib.check(lib.pysift_pca_basis_workspace_size(D, ctypes.byref(sz)), "pysift_pca_basis_workspace_size")
            wsb = torch.empty(int(sz.value), dtype=torch.uint8, device=self.device)
            _lib.check(lib.pysift_pca_basis(cov.data_ptr(), D, P, wsb.data_ptr(), wsb.numel(), proj.data_ptr(), None,
                                            st), "pysift_pca_basis")
            self._pca_matrix = proj
            self._pca_mean = mean
        if self.int8_matching:
            outf = torch.empty((n1 + n2, P), dtype=torch.float32, device=self.device)
            _lib.check(lib.pysift_pca_project_f32(both.data_ptr(), n1 + n2, D, self._pca_mean.data_ptr(),
                                                  self._pca_matrix.data_ptr(), P, outf.data_ptr(), st),
                       "pysift_pca_project_f32")
            return self._quantize(outf[:n1], outf[n1:])
        out = torch.empty((n1 + n2, P), dtype=torch.float16, device=self.device)
        _lib.check(lib.pysift_pca_project_f16(both.data_ptr(), n1 + n2, D, self._pca_mean.data_ptr(),
                                              self._pca_matrix.data_ptr(), P, out.data_ptr(), st),
                   "pysift_pca_project_f16")
        return ("f16", out[:n1], out[n1:])

    def _quantize(self, f1, f2):
        """int8 rows and scales of both sets (each quantised on its own, as
        pysift/core.py:2906-2907 does)."""
        from . import match
        st = torch.cuda.current_stream(self.device)
        q1, s1 = match.quantize_i8(f1, stream=st)
        q2, s2 = match.quantize_i8(f2, stream=st)
        return ("i8", q1, s1, q2, s2)

    def _match_prepared(self, prep, stream=None):
        from . import match
        if prep[0] == "i8":
            return match.match_i8(*prep[1:], self.match_ratio, stream=stream)
        return match.match_fp16(prep[1], prep[2], self.match_ratio, stream=stream)

    def _match(self, d1, d2):
        return self._match_prepared(self._prepare(d1, d2))

    def _random_stream(self, n_hyp):
        r = self._rand.get(n_hyp)
        if r is None:
            host = np.empty(4 * n_hyp, dtype=np.uint32)
            self._lib.pysift_mt19937_u32(42, host.ctypes.data_as(ctypes.c_void_p), host.size)
            r = torch.from_numpy(host).to(self.device)
            self._rand[n_hyp] = r
        return r

    def _ransac(self, p1, p2, n, key=""):
        st = self._stream()
        n_hyp = int(self.ransac_iters)
        sz = ctypes.c_size_t()
        _lib.check(self._lib.pysift_ransac_workspace_size(n, n_hyp, ctypes.byref(sz)), "ransac ws")
        ws = self._dev.get(key + "ransac_ws", (int(sz.value) + 256,), torch.uint8, self.device)
        wp, wn = _ptr_aligned(ws)
        H = self._dev.get(key + "ransac_H", (9,), torch.float64, self.device)
        mask = self._dev.get(key + "ransac_mask", (max(n, 1),), torch.uint8, self.device)
        info = self._dev.get(key + "ransac_info", (4,), torch.int32, self.device)
        rnd = self._random_stream(n_hyp)
        _lib.check(self._lib.pysift_ransac(p1.data_ptr(), p2.data_ptr(), n, rnd.data_ptr(), n_hyp,
                                           float(self.inlier_thresh), float(self.sigma_max),
                                           1 if self.ransac_method == 'magsac' else 0, 10, wp, wn, H.data_ptr(),
                                           mask.data_ptr(), info.data_ptr(), st), "pysift_ransac")
        return H, mask[:n], info

    def _match_and_ransac_launches(self, kp1, d1, n1, kp2, d2, n2):
        """Matcher preparation, matching, point gather and RANSAC of a pair,
        enqueued on the current stream with no host read: the match count
        stays on the device (RANSAC capacity: the smaller keypoint count)."""
        prep = self._prepare(d1, d2)
        self._mark(2)
        m = self._match_prepared(prep)
        self._mark(3)
        st = self._stream()
        cap = max(min(n1, n2), 1)
        # fresh buffers, not the instance's cached ones: under capture they
        # come from the graph's own memory pool, so a graph never writes
        # into a buffer that a later pair of another size replaced
        p1 = torch.empty((cap, 2), dtype=torch.float64, device=self.device)
        p2 = torch.empty((cap, 2), dtype=torch.float64, device=self.device)
        _lib.check(self._lib.pysift_gather_points(kp1.data_ptr(), m["pairs"].data_ptr(), m["count"].data_ptr(),
                                                  cap, 0, p1.data_ptr(), st), "gather")
        _lib.check(self._lib.pysift_gather_points(kp2.data_ptr(), m["pairs"].data_ptr(), m["count"].data_ptr(),
                                                  cap, 1, p2.data_ptr(), st), "gather")
        H_d, mask_d, info_d = self._ransac_count(p1, p2, m["count"], cap)
        self._mark(4)
        return m, p1, p2, H_d, mask_d, info_d

    #: graphs of the matcher + RANSAC stage kept per instance
    GRAPH_CACHE = 8

    def _match_and_ransac(self, kp1, d1, n1, kp2, d2, n2):
        """_match_and_ransac_launches as a CUDA graph replay: the first call
        for the keypoint counts and buffers runs eagerly (and fits the PCA
        basis on an instance's first pair) and captures the same launches,
        later calls replay them in one launch.
        Eager with stage_events (their records sit between the stages) or
        when the detector was built with graphs=False."""
        if not self._detector._use_graphs or self.stage_events is not None:
            return self._match_and_ransac_launches(kp1, d1, n1, kp2, d2, n2)
        key = ("pair", n1, n2, kp1.data_ptr(), d1.data_ptr(), kp2.data_ptr(), d2.data_ptr(), tuple(d1.shape[1:]),
               d1.dtype, self.pca_dims, self.int8_matching, self.ransac_iters, self.ransac_method,
               self.inlier_thresh, self.sigma_max, self.match_ratio)
        main = torch.cuda.current_stream(self.device)
        ent = self._graphs.get(key)
        if ent is None:
            out = self._match_and_ransac_launches(kp1, d1, n1, kp2, d2, n2)
            # at most GRAPH_CACHE graphs per instance (each holds its buffers
            # in its own memory pool); keys past that stay eager, so pairs of
            # many different sizes never recapture
            if len(self._graphs) >= self.GRAPH_CACHE:
                return out
            cap = self._capture_stream()
            cap.wait_stream(main)
            n0 = self._lib.pysift_launch_count()
            g = torch.cuda.CUDAGraph()
            outg = capture_graph(g, cap, lambda: self._match_and_ransac_launches(kp1, d1, n1, kp2, d2, n2))
            n = self._lib.pysift_launch_count() - n0
            self._lib.pysift_count_launches(-n)  # captured, not run
            self._graphs[key] = (g, outg, n)
            return out
        g, outg, n = ent
        with torch.cuda.stream(main):
            g.replay()
        self._lib.pysift_count_launches(n)
        return outg

    def _capture_stream(self):
        if getattr(self, "_cap_stream", None) is None:
            self._cap_stream = torch.cuda.Stream(self.device)
        return self._cap_stream

    def _ransac_count(self, p1, p2, count, cap):
        """_ransac with the point count on the device (up to `cap` points)."""
        st = self._stream()
        n_hyp = int(self.ransac_iters)
        sz = ctypes.c_size_t()
        _lib.check(self._lib.pysift_ransac_workspace_size(cap, n_hyp, ctypes.byref(sz)), "ransac ws")
        # fresh buffers (see _match_and_ransac_launches): a workspace freed
        # after a capture stays in that graph's private pool, which nothing
        # outside the capture allocates from
        ws = torch.empty((int(sz.value) + 256,), dtype=torch.uint8, device=self.device)
        wp, wn = _ptr_aligned(ws)
        H = torch.empty((9,), dtype=torch.float64, device=self.device)
        mask = torch.empty((cap,), dtype=torch.uint8, device=self.device)
        info = torch.empty((4,), dtype=torch.int32, device=self.device)
        rnd = self._random_stream(n_hyp)
        _lib.check(self._lib.pysift_ransac_count(p1.data_ptr(), p2.data_ptr(), count.data_ptr(), cap, rnd.data_ptr(),
                                                 n_hyp, float(self.inlier_thresh), float(self.sigma_max),
                                                 1 if self.ransac_method == 'magsac' else 0, 10, wp, wn,
                                                 H.data_ptr(), mask.data_ptr(), info.data_ptr(), st),
                   "pysift_ransac_count")
        return H, mask, info

    def _pinned(self, key, shape, dtype):
        """A cached page-locked host buffer."""
        t = self._dev.bufs.get(key)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, pin_memory=True)
            self._dev.bufs[key] = t
        return t

    @staticmethod
    def _compute_canvas_size(img1_shape, img2_shape, H):
        """pysift/core.py:3171-3187 (float64, host)."""
        h1, w1 = img1_shape[:2]
        h2, w2 = img2_shape[:2]
        c1 = np.array([[0, 0, 1], [w1, 0, 1], [w1, h1, 1], [0, h1, 1]], dtype=np.float64).T
        wc = H @ c1
        wc /= wc[2]
        ax = np.concatenate([wc[0], [0, w2, w2, 0]])
        ay = np.concatenate([wc[1], [0, 0, h2, h2]])
        ox = max(0.0, -ax.min())
        oy = max(0.0, -ay.min())
        return int(np.ceil(ax.max() + ox)) + 1, int(np.ceil(ay.max() + oy)) + 1, ox, oy

    def _compose_enqueue(self, img1, img2, H, key="", max_canvas_px=400_000_000):
        """Canvas geometry on the host, then warp, composition and the
        coverage extents on the current stream; the extents (and the seam
        RMSE) are copied to pinned host memory (read them after the stream
        has finished)."""
        hs, ws = img1.shape[:2]
        h2, w2 = img2.shape[:2]
        cw, ch, ox, oy = self._compute_canvas_size(img1.shape, img2.shape, H)
        if cw * ch > max_canvas_px or cw <= 0 or ch <= 0:
            raise RuntimeError(f"degenerate homography: canvas {cw}x{ch}")
        hinv = np.linalg.inv(H).astype(np.float32).ravel()
        iox, ioy = int(round(ox)), int(round(oy))
        st = self._stream()
        dev = self.device
        out = self._dev.get(key + "pano", (ch, cw, 3), torch.uint8, dev)
        ext = self._dev.get(key + "extents", (2 * ch + 2 * cw,), torch.int32, dev)
        hb = (ctypes.c_float * 9)(*[float(v) for v in hinv])
        multiband = self.blend == 'multiband' and cw > 1 and ch > 1
        if multiband:
            warped = self._dev.get(key + "warped1", (ch, cw, 3), torch.uint8, dev)
            m1 = self._dev.get(key + "mask1", (ch, cw), torch.uint8, dev)
            m2 = self._dev.get(key + "mask2", (ch, cw), torch.uint8, dev)
            outs = (None, warped.data_ptr(), m1.data_ptr(), m2.data_ptr())
        else:
            outs = (out.data_ptr(), None, None, None)
        _lib.check(self._lib.pysift_warp_feather(img1.data_ptr(), hs, ws, img1.stride(0), img2.data_ptr(), h2, w2,
                                                 img2.stride(0), cw, ch, ctypes.cast(hb, ctypes.c_void_p),
                                                 float(np.float32(ox)), float(np.float32(oy)), iox, ioy, 1, *outs,
                                                 ext.data_ptr(), ext[ch:].data_ptr(), ext[2 * ch:].data_ptr(),
                                                 ext[2 * ch + cw:].data_ptr(), st), "pysift_warp_feather")
        res = dict(out=out, canvas_w=cw, canvas_h=ch, ox=ox, oy=oy, seam_rmse_host=None)
        if multiband:
            from . import blend as _blend
            canvas2 = self._dev.get(key + "canvas2", (ch, cw, 3), torch.uint8, dev)
            _lib.check(self._lib.pysift_place_image(img2.data_ptr(), h2, w2, img2.stride(0), cw, ch, iox, ioy,
                                                    canvas2.data_ptr(), None, st), "pysift_place_image")
            need = _blend.workspace_bytes(cw, ch, self.n_blend_levels) + 256
            wsb = self._dev.get(key + "blend_ws", (need,), torch.uint8, dev)
            both = self._dev.get(key + "both", (ch, cw), torch.uint8, dev)
            rmse = self._dev.get(key + "seam_rmse", (1,), torch.float64, dev)
            _blend.blend_multiband(warped, m1, canvas2, m2, self.n_blend_levels, color_match=self.color_match,
                                   workspace=wsb, pano=out,
                                   both=both, seam_rmse=rmse, stream=st)
            rmse_host = torch.empty(1, dtype=torch.float64, pin_memory=True)
            rmse_host.copy_(rmse, non_blocking=True)
            res.update(seam_rmse_host=rmse_host, warped1=warped, mask1=m1, mask2=m2, canvas2=canvas2)
        ext_host = torch.empty(ext.shape, dtype=torch.int32, pin_memory=True)
        ext_host.copy_(ext, non_blocking=True)
        res["ext_host"] = ext_host
        return res

    def _compose_crop(self, c):
        """The inner-rectangle crop of a composed canvas (its extents on the
        host; pysift_autocrop_box): a device view of the canvas."""
        cw, ch, out = c["canvas_w"], c["canvas_h"], c["out"]
        e = np.ascontiguousarray(c["ext_host"].numpy(), dtype=np.int32)
        box = np.empty(5, dtype=np.int32)
        p = e.ctypes.data
        _lib.check(self._lib.pysift_autocrop_box(p, p + 4 * ch, p + 8 * ch, p + 8 * ch + 4 * cw, cw, ch,
                                                 box.ctypes.data), "pysift_autocrop_box")
        x, y, w, h = (int(v) for v in box[:4])
        c["crop_box"] = (x, y, w, h)
        return out[y:y + h, x:x + w]

    def _compose(self, img1, img2, H, max_canvas_px=400_000_000):
        c = self._compose_enqueue(img1, img2, H, max_canvas_px=max_canvas_px)
        torch.cuda.current_stream(self.device).synchronize()
        pano = self._to_host(self._compose_crop(c))
        self._last_compose = c
        return pano, dict(canvas_w=c["canvas_w"], canvas_h=c["canvas_h"], ox=c["ox"], oy=c["oy"],
                          seam_rmse=self._seam_rmse_of(c), crop_box=c.get("crop_box"))

    @staticmethod
    def _seam_rmse_of(c):
        r = c.get("seam_rmse_host")
        return float(r[0]) if r is not None else float('nan')

    def _to_host(self, t):
        """Device tensor -> numpy array in page-locked memory from torch's
        caching host allocator (the array keeps its block alive; a freed
        block is reused by a later call)."""
        host = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        if t.dim() >= 2 and not t.is_contiguous() and t[0].is_contiguous() and t.numel() > 0:
            # rows of a crop: one strided copy, no packing launch
            rb = t[0].numel() * t.element_size()
            _lib.check(self._lib.pysift_copy2d(host.data_ptr(), rb, t.data_ptr(), t.stride(0) * t.element_size(),
                                               rb, t.shape[0], self._stream()), "pysift_copy2d")
        else:
            host.copy_(t.contiguous(), non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return host.numpy()

    # ------------------------------------------------------------------
    def _stitch_pair(self, img1, img2):
        """pysift/core.py:3720-3818 (two images, img2 is the reference frame)."""
        timings, metrics = {}, {}
        with torch.cuda.device(self.device):
            t0 = time.perf_counter()
            self._mark(0)
            # the two views run concurrently, one side stream each
            main = torch.cuda.current_stream(self.device)
            if self._side is None:
                self._side = (torch.cuda.Stream(self.device), torch.cuda.Stream(self.device))
            s1, s2 = self._side
            s1.wait_stream(main)
            s2.wait_stream(main)
            g1, b1 = self._detect_view(img1, "img1", 0, s1)
            g2, b2 = self._detect_view(img2, "img2", 1, s2)
            s1.synchronize()
            s2.synchronize()
            main.wait_stream(s1)
            main.wait_stream(s2)
            self._mark(1)
            kp1, d1, n1 = self._select(b1, "img1")
            kp2, d2, n2 = self._select(b2, "img2")
            metrics.update(kp1=n1, kp2=n2)
            if n1 == 0 or n2 < 2:
                raise RuntimeError(f"Insufficient matches (0), need >= 4")
            m, p1, p2, H_d, mask_d, info_d = self._match_and_ransac(kp1, d1, n1, kp2, d2, n2)
            timings['st1'] = time.perf_counter() - t0
            timings['st2'] = 0.0
            t0 = time.perf_counter()
            hh = self._pinned("ransac_H_host", (9,), torch.float64)
            ih = self._pinned("ransac_info_host", (4,), torch.int32)
            ch = self._pinned("match_count_host", (1,), torch.int32)
            hh.copy_(H_d, non_blocking=True)
            ih.copy_(info_d, non_blocking=True)
            ch.copy_(m["count"][:1], non_blocking=True)
            torch.cuda.current_stream(self.device).synchronize()
            H = hh.numpy().reshape(3, 3).copy()
            info = ih.numpy()[:3].copy()
            n_m, n_in = int(ch.numpy()[0]), int(info[0])
            metrics.update(matches=n_m)
            timings['st3'] = time.perf_counter() - t0
            if n_m < 4:
                raise RuntimeError(f"Insufficient matches ({n_m}), need >= 4")
            mask_d = mask_d[:n_m]
            p1, p2 = p1[:n_m], p2[:n_m]
            metrics.update(inliers=n_in, inlier_ratio=n_in / max(n_m, 1))
            if n_in < 4:
                raise RuntimeError(f"Only {n_in} inliers after RANSAC, need >= 4")
            timings['st4'] = 0.0
            metrics.update(depth_cv=None, bands=self.n_depth_layers)
            t0 = time.perf_counter()
            pano, cm = self._compose(g1, g2, H)
            self._mark(5)
            timings['st5'] = time.perf_counter() - t0
            metrics.update(canvas_w=cm['canvas_w'], canvas_h=cm['canvas_h'], seam_rmse=cm['seam_rmse'],
                           crop_box=cm['crop_box'])
        self._last = dict(H=H, mask=mask_d, pairs=m["pairs"][:n_m], kp1=kp1, kp2=kp2, p1=p1, p2=p2, info=info)
        return pano, timings, metrics

    @staticmethod
    def _compute_canvas_size_3(img1_shape, img2_shape, img3_shape, H12, H32):
        """pysift/core.py:3190-3208 (float64, host)."""
        h2, w2 = img2_shape[:2]
        all_x = [0.0, float(w2), float(w2), 0.0]
        all_y = [0.0, 0.0, float(h2), float(h2)]
        for shp, H in ((img1_shape, H12), (img3_shape, H32)):
            h, w = shp[:2]
            c = np.array([[0, 0, 1], [w, 0, 1], [w, h, 1], [0, h, 1]], dtype=np.float64).T
            wc = H @ c
            wc /= wc[2]
            all_x.extend(wc[0].tolist())
            all_y.extend(wc[1].tolist())
        ax, ay = np.array(all_x), np.array(all_y)
        ox = max(0.0, -ax.min())
        oy = max(0.0, -ay.min())
        return int(np.ceil(ax.max() + ox)) + 1, int(np.ceil(ay.max() + oy)) + 1, ox, oy

    def _verify_chain(self, H_AB, H_CB):
        """pysift/core.py:3564-3586: rotation and scale of inv(H_CB) H_AB,
        printed with a warning past 5 degrees or 15 % (when verbose); returned
        as metrics chain_rotation_deg / chain_scale."""
        try:
            Hc = np.linalg.inv(H_CB) @ H_AB
            Hc /= Hc[2, 2]
        except np.linalg.LinAlgError:
            if self.verbose:
                print("  [Chain] WARNING: H_CB is singular")
            return {}
        theta = float(np.degrees(np.arctan2(Hc[1, 0], Hc[0, 0])))
        scale = float(np.sqrt(abs(np.linalg.det(Hc[:2, :2]))))
        if self.verbose:
            warns = []
            if abs(theta) > 5.0:
                warns.append(f"rotation drift {theta:+.1f} deg")
            if abs(scale - 1.0) > 0.15:
                warns.append(f"scale drift {scale:.3f}x")
            status = "OK" if not warns else "WARN: " + ", ".join(warns)
            print(f"  [Chain] rotation={theta:+.1f} deg scale={scale:.3f}  [{status}]")
        return dict(chain_rotation_deg=theta, chain_scale=scale)

    def _warp_to_canvas(self, img, H, ref, cw, ch, ox, oy, key):
        """Warped uint8 image and mask of `img` on the canvas (the warp of
        pysift/core.py:3210-3239); `ref` is the reference view the kernel
        places (its outputs are not used here)."""
        hs, ws = img.shape[:2]
        hinv = np.linalg.inv(H).astype(np.float32).ravel()
        hb = (ctypes.c_float * 9)(*[float(v) for v in hinv])
        warped = self._dev.get(key + "warped", (ch, cw, 3), torch.uint8, self.device)
        mask = self._dev.get(key + "mask", (ch, cw), torch.uint8, self.device)
        _lib.check(self._lib.pysift_warp_feather(img.data_ptr(), hs, ws, img.stride(0), ref.data_ptr(), ref.shape[0],
                                                 ref.shape[1], ref.stride(0), cw, ch, ctypes.cast(hb, ctypes.c_void_p),
                                                 float(np.float32(ox)), float(np.float32(oy)), int(round(ox)),
                                                 int(round(oy)), 0, None, warped.data_ptr(), mask.data_ptr(), None,
                                                 None, None, None, None, self._stream()), "pysift_warp_feather")
        return warped, mask

    def _stitch_triple(self, img1, img2, img3):
        """pysift/core.py:3820-3966 (three images, img2 is the reference
        frame): features of all three views, matches 1-2 and 2-3 (the PCA
        basis fitted on the first pair), RANSAC 1->2 and 3->2, one canvas,
        then the two-pass composition: image 1 blended with image 2, the
        unclipped float result blended with image 3, paste and crop."""
        if self.blend != 'multiband':
            raise NotImplementedError("three-image stitching composes with the reference's multiband blend only")
        from . import blend as _blend
        timings, metrics = {}, {}
        with torch.cuda.device(self.device):
            t0 = time.perf_counter()
            main = torch.cuda.current_stream(self.device)
            if self._side is None:
                self._side = (torch.cuda.Stream(self.device), torch.cuda.Stream(self.device))
            if not hasattr(self, "_side3"):
                self._side3 = torch.cuda.Stream(self.device)
            streams = (self._side[0], self._side[1], self._side3)
            for s_ in streams:
                s_.wait_stream(main)
            views = [self._detect_view(img, f"img{i + 1}", i, s_) for i, (img, s_) in
                     enumerate(zip((img1, img2, img3), streams))]
            for s_ in streams:
                s_.synchronize()
                main.wait_stream(s_)
            (g1, b1), (g2, b2), (g3, b3) = views
            kp1, d1, n1 = self._select(b1, "img1")
            kp2, d2, n2 = self._select(b2, "img2")
            kp3, d3, n3 = self._select(b3, "img3")
            metrics.update(kp1=n1, kp2=n2, kp3=n3)
            if min(n1, n2, n3) < 2:
                raise RuntimeError("Insufficient matches for 3-image stitching")
            m12 = self._match_prepared(self._prepare(d1, d2))
            m23 = self._match_prepared(self._prepare(d2, d3))
            c12, c23 = (int(v) for v in torch.cat([m12["count"], m23["count"]]).cpu().numpy())
            metrics.update(matches_12=c12, matches_23=c23)
            timings['st1'] = time.perf_counter() - t0
            if c12 < 4 or c23 < 4:
                raise RuntimeError("Insufficient matches for 3-image stitching")
            st = self._stream()

            def gather(kp, m, n, side):
                p = torch.empty((n, 2), dtype=torch.float64, device=self.device)
                _lib.check(self._lib.pysift_gather_points(kp.data_ptr(), m["pairs"].data_ptr(), m["count"].data_ptr(),
                                                          n, side, p.data_ptr(), st), "gather")
                return p

            pA, pB1 = gather(kp1, m12, c12, 0), gather(kp2, m12, c12, 1)
            pB2, pC = gather(kp2, m23, c23, 0), gather(kp3, m23, c23, 1)
            timings['st2'] = 0.0
            t0 = time.perf_counter()
            H12_d, _, info12 = self._ransac(pA, pB1, c12, key="t12_")
            H32_d, _, info32 = self._ransac(pC, pB2, c23, key="t32_")
            Hs = torch.stack([H12_d, H32_d]).cpu().numpy().reshape(2, 3, 3)
            infos = torch.stack([info12, info32]).cpu().numpy()
            H12, H32 = Hs[0].copy(), Hs[1].copy()
            timings['st3'] = time.perf_counter() - t0
            metrics.update(inliers_12=int(infos[0][0]), inliers_32=int(infos[1][0]))
            if min(int(infos[0][0]), int(infos[1][0])) < 4:
                raise RuntimeError("Too few inliers for 3-image stitching")
            metrics.update(self._verify_chain(H12, H32))
            timings['st4'] = 0.0
            metrics.update(depth_cv=None, bands=self.n_depth_layers)
            t0 = time.perf_counter()
            cw, ch, ox, oy = self._compute_canvas_size_3(g1.shape, g2.shape, g3.shape, H12, H32)
            if cw * ch > 400_000_000 or cw <= 1 or ch <= 1:
                raise RuntimeError(f"degenerate homography: canvas {cw}x{ch}")
            w1, mk1 = self._warp_to_canvas(g1, H12, g2, cw, ch, ox, oy, "t1_")
            w3, mk3 = self._warp_to_canvas(g3, H32, g2, cw, ch, ox, oy, "t3_")
            canvas2 = self._dev.get("t2_canvas", (ch, cw, 3), torch.uint8, self.device)
            mk2 = self._dev.get("t2_mask", (ch, cw), torch.uint8, self.device)
            _lib.check(self._lib.pysift_place_image(g2.data_ptr(), g2.shape[0], g2.shape[1], g2.stride(0), cw, ch,
                                                    int(round(ox)), int(round(oy)), canvas2.data_ptr(),
                                                    mk2.data_ptr(), st), "pysift_place_image")
            need = _blend.workspace_bytes(cw, ch, self.n_blend_levels) + 256
            wsb = self._dev.get("t_blend_ws", (need,), torch.uint8, self.device)
            b12 = self._dev.get("t_b12", (ch, cw, 3), torch.float32, self.device)
            m12u = self._dev.get("t_m12", (ch, cw), torch.uint8, self.device)
            r12 = self._dev.get("t_r12", (1,), torch.float64, self.device)
            _blend.blend_multiband(w1, mk1, canvas2, mk2, self.n_blend_levels, color_match=self.color_match,
                                   workspace=wsb, both=m12u,
                                   seam_rmse=r12, blended=b12, want_pano=False, stream=st)
            pano = self._dev.get("t_pano", (ch, cw, 3), torch.uint8, self.device)
            both = self._dev.get("t_both", (ch, cw), torch.uint8, self.device)
            r23 = self._dev.get("t_r23", (1,), torch.float64, self.device)
            _blend.blend_multiband(b12, m12u, w3, mk3, self.n_blend_levels, color_match=self.color_match,
                                   workspace=wsb, pano=pano, both=both,
                                   seam_rmse=r23, stream=st)
            ext = _blend.mask_extents(both, out=self._dev.get("t_ext", (2 * ch + 2 * cw,), torch.int32, self.device),
                                      stream=st)
            e = ext.cpu().numpy()
            rmse = torch.cat([r12, r23]).cpu().numpy()
            crop = self._compose_crop(dict(out=pano, canvas_w=cw, canvas_h=ch, ext_host=torch.from_numpy(e)))
            pano_h = self._to_host(crop)
            timings['st5'] = time.perf_counter() - t0
            metrics.update(seam_rmse=float(rmse[0]), seam_rmse_23=float(rmse[1]), canvas_w=cw, canvas_h=ch)
        self._last = dict(H12=H12, H32=H32, info12=infos[0], info32=infos[1], pairs12=m12["pairs"][:c12],
                          pairs23=m23["pairs"][:c23], warped1=w1, mask1=mk1, warped3=w3, mask3=mk3, canvas2=canvas2,
                          mask2=mk2, ox=ox, oy=oy)
        return pano_h, timings, metrics

    def _side_streams(self, n):
        if not hasattr(self, "_batch_streams"):
            self._batch_streams = []
        while len(self._batch_streams) < n:
            self._batch_streams.append(torch.cuda.Stream(self.device))
        return self._batch_streams[:n]

    def stitch_batch(self, pairs, n_streams=8):
        """Stitch many two-image pairs in one call; returns the panoramas in
        input order.  Each phase runs for all pairs at once, spread over
        `n_streams` CUDA streams, with one host synchronisation per phase:
        (1) CLAHE and detection of every view, (2) matcher preparation and
        matching, (3) RANSAC, (4) warp + composition, crop and readback.
        Every pair gets exactly the result stitch(img1, img2) gives on this
        instance; the PCA basis is fitted on the first pair if it is not yet
        fitted.  No file is written.  The per-pair metrics are kept in
        last_batch_metrics."""
        from . import match as _match_mod
        P = len(pairs)
        if P == 0:
            return []
        ns = max(1, min(int(n_streams), 2 * P))
        with torch.cuda.device(self.device):
            main = torch.cuda.current_stream(self.device)
            streams = self._side_streams(ns)
            for s in streams:
                s.wait_stream(main)
            # (1) features
            bgrs, grays = [], []
            pairs = [tuple(self._preprocess_image(im) for im in pr) for pr in pairs]
            for p, pr in enumerate(pairs):
                if len(pr) != 2:
                    raise ValueError("stitch_batch takes (img1, img2) pairs")
                for v in range(2):
                    st = streams[(2 * p + v) % ns]
                    with torch.cuda.stream(st):
                        key = f"b{p}_{v}"
                        bgr = self._upload_bgr(pr[v], key)
                        bgrs.append(bgr)
                        grays.append(self._gray_clahe(bgr, key))
            for s in streams:
                main.wait_stream(s)
            feats = self._detector.detect_batch(grays, n_streams=ns, gpu_output=True)
            metrics = [dict(kp1=int(feats[2 * p][0].shape[0]), kp2=int(feats[2 * p + 1][0].shape[0]))
                       for p in range(P)]
            for p, m in enumerate(metrics):
                if m["kp1"] == 0 or m["kp2"] < 2:
                    raise RuntimeError(f"pair {p}: Insufficient matches (0), need >= 4")
            # (2) preparation + matching (the PCA basis from the first pair, as stitch() does)
            if self._pca_matrix is None:
                self._prepare(feats[0][1], feats[1][1])
            for s in streams:
                s.wait_stream(main)
            matches = []
            for p in range(P):
                st = streams[p % ns]
                with torch.cuda.stream(st):
                    prep = self._prepare(feats[2 * p][1], feats[2 * p + 1][1])
                    matches.append(self._match_prepared(prep, stream=st))
            for s in streams:
                main.wait_stream(s)
            counts = torch.cat([m["count"] for m in matches]).cpu().numpy()
            # (3) RANSAC
            for s in streams:
                s.wait_stream(main)
            rs = []
            for p in range(P):
                n_m = int(counts[p])
                metrics[p]["matches"] = n_m
                if n_m < 4:
                    raise RuntimeError(f"pair {p}: Insufficient matches ({n_m}), need >= 4")
                st = streams[p % ns]
                with torch.cuda.stream(st):
                    sst = st.cuda_stream
                    p1 = torch.empty((n_m, 2), dtype=torch.float64, device=self.device)
                    p2 = torch.empty((n_m, 2), dtype=torch.float64, device=self.device)
                    m = matches[p]
                    _lib.check(self._lib.pysift_gather_points(feats[2 * p][0].data_ptr(), m["pairs"].data_ptr(),
                                                              m["count"].data_ptr(), n_m, 0, p1.data_ptr(), sst),
                               "gather")
                    _lib.check(self._lib.pysift_gather_points(feats[2 * p + 1][0].data_ptr(), m["pairs"].data_ptr(),
                                                              m["count"].data_ptr(), n_m, 1, p2.data_ptr(), sst),
                               "gather")
                    rs.append(self._ransac(p1, p2, n_m, key=f"b{p}_"))
            for s in streams:
                main.wait_stream(s)
            Hs = torch.stack([r[0] for r in rs]).cpu().numpy().reshape(P, 3, 3)
            infos = torch.stack([r[2] for r in rs]).cpu().numpy()
            # (4) compose
            for s in streams:
                s.wait_stream(main)
            comps = []
            for p in range(P):
                n_in = int(infos[p][0])
                metrics[p].update(inliers=n_in)
                if n_in < 4:
                    raise RuntimeError(f"pair {p}: Only {n_in} inliers after RANSAC, need >= 4")
                st = streams[p % ns]
                with torch.cuda.stream(st):
                    comps.append(self._compose_enqueue(bgrs[2 * p], bgrs[2 * p + 1], Hs[p].copy(), key=f"b{p}_"))
                metrics[p].update(canvas_w=comps[p]["canvas_w"], canvas_h=comps[p]["canvas_h"])
            for s in streams:
                main.wait_stream(s)
            main.synchronize()
            for p, c in enumerate(comps):
                metrics[p]["seam_rmse"] = self._seam_rmse_of(c)
            hosts = []
            for c in comps:
                crop = self._compose_crop(c).contiguous()
                host = torch.empty(crop.shape, dtype=crop.dtype, pin_memory=True)
                host.copy_(crop, non_blocking=True)
                hosts.append(host)
            main.synchronize()
        self.last_batch_metrics = metrics
        self._last_batch_H = Hs
        return [h.numpy() for h in hosts]

    def stitch(self, *args):
        """Stitch two or three images (pysift/core.py:3972-4008; with three, the
        middle one is the reference frame); returns the BGR uint8
        panorama and, as the reference does, writes panorama_<ts>.png to the
        working directory unless the instance was built with save_output=False."""
        if len(args) == 1 and isinstance(args[0], (list, tuple)):
            images = list(args[0])
        else:
            images = list(args)
        if len(images) in (2, 3):
            images = [self._preprocess_image(im) for im in images]
        if len(images) == 2:
            pano, timings, metrics = self._stitch_pair(images[0], images[1])
        elif len(images) == 3:
            pano, timings, metrics = self._stitch_triple(images[0], images[1], images[2])
        else:
            raise ValueError(f"stitch() accepts 2 or 3 images, got {len(images)}")
        self.last_timings, self.last_metrics = timings, metrics
        if self.verbose:
            if len(images) == 2:
                print(f"[pysift_b200] kp {metrics['kp1']}/{metrics['kp2']}  matches {metrics['matches']}  "
                      f"inliers {metrics['inliers']}  canvas {metrics['canvas_w']}x{metrics['canvas_h']}")
            else:
                print(f"[pysift_b200] kp {metrics['kp1']}/{metrics['kp2']}/{metrics['kp3']}  matches "
                      f"{metrics['matches_12']}/{metrics['matches_23']}  inliers {metrics['inliers_12']}/"
                      f"{metrics['inliers_32']}  canvas {metrics['canvas_w']}x{metrics['canvas_h']}")
        if self.save_output:
            import cv2
            out = self._postprocess(pano)
            ts = datetime.now().strftime("%Y%m%d_%H%M%S")
            ext = 'jpg' if self.output_format in ('jpg', 'jpeg') else 'png'
            fname = f"panorama_{ts}.{ext}"
            if ext == 'jpg':
                cv2.imwrite(fname, out, [cv2.IMWRITE_JPEG_QUALITY, self.output_quality])
            else:
                cv2.imwrite(fname, out)
        return pano

    def _preprocess_image(self, img):
        """The reference's optional preprocessing of each input
        (pysift/core.py:2486-2514), with its own OpenCV calls on host images:
        resize the longest side to max_dimension (INTER_AREA), bilateral
        filter (denoise), unsharp mask (sharpen).  CUDA tensor inputs take no
        preprocessing options."""
        if not (self.max_dimension > 0 or self.denoise or self.sharpen):
            return img
        if isinstance(img, torch.Tensor):
            raise NotImplementedError("max_dimension / denoise / sharpen apply to host (numpy) images only")
        import cv2
        if self.max_dimension > 0:
            h, w = img.shape[:2]
            scale = self.max_dimension / max(h, w)
            if scale < 1.0:
                nw, nh = int(w * scale), int(h * scale)
                img = cv2.resize(img, (nw, nh), interpolation=cv2.INTER_AREA)
                if self.verbose:
                    print(f"    Resized {w}x{h} -> {nw}x{nh}  (scale {scale:.2f})")
        if self.denoise:
            img = cv2.bilateralFilter(img, d=9, sigmaColor=75, sigmaSpace=75)
        if self.sharpen:
            blur = cv2.GaussianBlur(img, (0, 0), sigmaX=2.0)
            img = cv2.addWeighted(img, 1.5, blur, -0.5, 0)
        return np.ascontiguousarray(img)

    def _postprocess(self, pano):
        """The reference's post-processing of the saved panorama
        (pysift/core.py:4054-4075): resize the longest side to output_max_dim
        (INTER_AREA), unsharp mask (post_sharpen).  The returned panorama is
        not post-processed, as in the reference."""
        if not (self.output_max_dim > 0 or self.post_sharpen):
            return pano
        import cv2
        if self.output_max_dim > 0:
            h, w = pano.shape[:2]
            scale = self.output_max_dim / max(h, w)
            if scale < 1.0:
                pano = cv2.resize(pano, (int(w * scale), int(h * scale)), interpolation=cv2.INTER_AREA)
        if self.post_sharpen:
            blur = cv2.GaussianBlur(pano, (0, 0), sigmaX=2.0)
            pano = cv2.addWeighted(pano, 1.5, blur, -0.5, 0)
        return pano
