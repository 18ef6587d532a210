"""PySIFT / GPUPyStitch drop-in classes backed by libpysift_b200.so.

Mirrors the public surface of the reference (pysift/core.py of
SivaIITM/PySIFT): the same class names, constructor keyword arguments and
defaults, ``detectAndCompute(gray, mask=None, profile=False, gpu_output=False)``
and ``stitch(*imgs)``.  The detection pipeline runs as one C-ABI call
(pysift_detect_and_compute) on the current torch CUDA stream; torch supplies
device memory, streams and pinned host buffers.
"""
import ctypes
import math
import time

import numpy as np
import torch

from . import _lib

_GIB = 1024 ** 3

# pysift/core.py:1198-1202
DSP_PRESETS = {
    3: np.array([1.0 / math.sqrt(2), 1.0, math.sqrt(2)], dtype=np.float32),
    4: np.array([0.5, 1.0 / math.sqrt(2), 1.0, math.sqrt(2)], dtype=np.float32),
    5: np.array([0.5, 1.0 / math.sqrt(2), 1.0, math.sqrt(2), 2.0], dtype=np.float32),
}

MAX_CANDS_PER_OCTAVE = 25000   # pysift/core.py:1395
KEYPOINT_CAP = 8000             # pysift/core.py:2078
STARVATION_MIN = 100            # pysift/core.py:2066
BORDER = 5                      # pysift/core.py:1381


def _device_high_vram(device):
    """The reference's tier switch (pysift/core.py:114): >= 12 GB of VRAM."""
    props = torch.cuda.get_device_properties(device)
    return props.total_memory / _GIB >= 12


def capture_graph(g, stream, fn):
    """Capture the launches fn() enqueues on `stream` into CUDA graph `g` and
    return fn()'s result.  Unlike the torch.cuda.graph context manager this
    neither synchronizes nor empties the device and pinned-host allocator
    caches, so a capture in the middle of a run of varying image sizes does
    not send the calls after it back to cudaMalloc and cudaHostAlloc."""
    with torch.cuda.stream(stream):
        g.capture_begin()
        try:
            return fn()
        finally:
            g.capture_end()


def gaussian_weights(sigma, truncate=4):
    """1-D Gaussian weights exactly as pysift/core.py:563-577 computes them
    (numpy float32); radius 0 when sigma < 0.01 (no blur)."""
    if sigma < 0.01:
        return np.ones(1, np.float32), 0
    radius = int(truncate * sigma + 0.5)
    x = np.arange(-radius, radius + 1, dtype=np.float32)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    return k.astype(np.float32), radius


def check_detector_options(dsp_n_scales, orientation, descriptor):
    """Reject the detector options this backend does not carry, before any
    device work: the reference's DSP scale-count check
    (pysift/core.py:1203-1204), and the learned orientation and descriptor
    paths, which raise NotImplementedError instead of falling back."""
    if dsp_n_scales not in DSP_PRESETS:
        raise ValueError(f"dsp_n_scales must be 3, 4, or 5 (got {dsp_n_scales})")
    if orientation != 'histogram':
        raise NotImplementedError(
            f"orientation={orientation!r}: only the histogram orientation is implemented on this backend "
            "(the learned OriNet/AffNet paths are not part of it)")
    if descriptor != 'sift':
        raise NotImplementedError(
            f"descriptor={descriptor!r}: only the SIFT descriptor is implemented on this backend "
            "(the learned HardNet/HyNet paths are not part of it)")


def build_detect_config(n_octaves, n_scales, sigma0, contrast_thresh, edge_thresh, dsp, dsp_n_scales,
                        fp16_pyramid, double_image, rootsift, high_vram):
    """Fill pysift_detect_config the way the reference's host code derives
    its parameters (pysift/core.py:1234-1290, 1475-1477, 1540-1555,
    1790-1810, 1508-1521)."""
    cfg = _lib.DetectConfig()
    S = n_scales
    if S < 1 or S + 3 > _lib.MAX_LEVELS:
        raise ValueError(f"n_scales must be in 1..{_lib.MAX_LEVELS - 3}")
    if n_octaves < 1 or n_octaves > _lib.MAX_OCTAVES:
        raise ValueError(f"n_octaves must be in 1..{_lib.MAX_OCTAVES}")
    cfg.n_octaves = n_octaves
    cfg.n_scales = S
    cfg.sigma0 = sigma0
    cfg.contrast_thresh = contrast_thresh
    cfg.edge_score = float((edge_thresh + 1.0) ** 2 / edge_thresh)
    cfg.double_image = 1 if double_image else 0
    cfg.double_px_cap = 16_000_000 if high_vram else 4_194_304
    cfg.fp16_pyramid = 1 if fp16_pyramid else 0
    cfg.dsp = 1 if dsp else 0
    scales = DSP_PRESETS[dsp_n_scales]
    cfg.n_dsp = len(scales)
    for i, v in enumerate(scales):
        cfg.dsp_scales[i] = float(v)
    cfg.rootsift = 1 if rootsift else 0
    cfg.max_cands_per_octave = MAX_CANDS_PER_OCTAVE
    cfg.keypoint_cap = KEYPOINT_CAP
    cfg.starvation_min = STARVATION_MIN
    cfg.border = BORDER
    k = 2.0 ** (1.0 / S)
    sigmas = [sigma0 * (k ** s) for s in range(S + 3)]
    sd_double = float(np.sqrt(max(sigma0 ** 2 - 1.0 ** 2, 1e-6)))
    sd_single = float(np.sqrt(max(sigma0 ** 2 - 0.5 ** 2, 1e-6)))
    inc = [float(np.sqrt(max(sigmas[s] ** 2 - sigmas[s - 1] ** 2, 1e-6))) for s in range(1, S + 3)]
    for idx, sig in enumerate([sd_double, sd_single] + inc):
        w, r = gaussian_weights(sig, 4)
        if r > _lib.MAX_RADIUS:
            raise ValueError(f"Gaussian radius {r} exceeds {_lib.MAX_RADIUS}")
        cfg.blur_radius[idx] = r
        for j, v in enumerate(w):
            cfg.blur_weights[idx][j] = float(v)
    si = np.arange(_lib.MAX_LEVELS, dtype=np.float32)
    ori_sigma = (sigma0 * (k ** si)).astype(np.float32)                      # pysift/core.py:1555
    desc_ph = np.maximum(4.0, np.round(3.0 * sigma0 * (k ** si) * math.sqrt(2) * 2.5)).astype(np.float32)
    for s in range(_lib.MAX_LEVELS):
        cfg.ori_sigma[s] = float(ori_sigma[s])
        cfg.desc_ph[s] = float(desc_ph[s])
    for d, cs in enumerate([1.0, 0.5]):                                       # pysift/core.py:1508-1521
        for o in range(_lib.MAX_OCTAVES):
            for s in range(_lib.MAX_LEVELS):
                cfg.kp_size[d][o][s] = float(np.float32(sigma0 * (k ** s) * float(2 ** o) * cs * 2.0))
    return cfg


class _Buffers:
    """Device workspace and outputs for one image size (torch-allocated)."""

    def __init__(self, lib, cfg, H, W, device):
        size = ctypes.c_size_t(0)
        _lib.check(lib.pysift_detect_workspace_size(ctypes.byref(cfg), H, W, ctypes.byref(size)),
                   "pysift_detect_workspace_size")
        self.ws_bytes = int(size.value)
        self.ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=device)
        self.ws_off = (-self.ws.data_ptr()) % 256
        self.max_out = int(lib.pysift_detect_max_keypoints(ctypes.byref(cfg)))
        self.kpts = torch.empty((self.max_out, 4), dtype=torch.float32, device=device)
        self.resp = torch.empty(self.max_out, dtype=torch.float32, device=device)
        self.octv = torch.empty(self.max_out, dtype=torch.int32, device=device)
        self.desc = torch.empty((self.max_out, 128), dtype=torch.float32, device=device)
        self.stats = torch.zeros(_lib.STAT_COUNT, dtype=torch.int32, device=device)
        self.stats_host = torch.zeros(_lib.STAT_COUNT, dtype=torch.int32).pin_memory()
        self.gray = torch.empty((H, W), dtype=torch.uint8, device=device)
        self.gray_host = torch.empty((H, W), dtype=torch.uint8).pin_memory()

    @property
    def ws_ptr(self):
        return self.ws.data_ptr() + self.ws_off


class _BatchOutputs:
    """Output buffers of one image of a batch."""

    def __init__(self, max_out, device):
        self.kpts = torch.empty((max_out, 4), dtype=torch.float32, device=device)
        self.resp = torch.empty(max_out, dtype=torch.float32, device=device)
        self.octv = torch.empty(max_out, dtype=torch.int32, device=device)
        self.desc = torch.empty((max_out, 128), dtype=torch.float32, device=device)
        self.stats = torch.zeros(_lib.STAT_COUNT, dtype=torch.int32, device=device)
        self.stats_host = torch.zeros(_lib.STAT_COUNT, dtype=torch.int32).pin_memory()


def keypoints_from_rows(kp, resp, octv):
    """cv2.KeyPoint list from output rows [x, y, size, angle], response and
    octave (pysift/core.py:2139-2142), built by mapping the constructor over
    Python lists (about 3.5x faster than a per-row loop)."""
    import cv2
    c = np.asarray(kp, np.float64).T.tolist()
    return list(map(cv2.KeyPoint, c[0], c[1], c[2], c[3], np.asarray(resp, np.float64).tolist(),
                    np.asarray(octv).astype(np.int64).tolist()))


class PySIFT:
    """GPU SIFT detector/descriptor with the reference's interface
    (pysift/core.py:1150-2172).

    Not thread-safe: an instance keeps per-size device buffers and a pinned
    staging buffer, like the reference's instance (pysift/core.py:1217-1226).
    """

    def __init__(self, n_octaves=None, n_scales=3, sigma0=1.6, contrast_thresh=0.04, edge_thresh=10.0,
                 dsp=False, dsp_n_scales=3, fp16_pyramid=None, orientation='histogram', descriptor='sift',
                 double_image=True, rootsift=True, *, device=None, high_vram=None, as_uint8=False,
                 graphs=True):
        check_detector_options(dsp_n_scales, orientation, descriptor)
        if as_uint8 and rootsift:
            raise ValueError("as_uint8 converts the L2 / clip / L2 descriptor as OpenCV does: "
                             "construct with rootsift=False")
        if not torch.cuda.is_available():
            raise RuntimeError("PySIFT (pysift_b200) needs a CUDA device")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        hv = _device_high_vram(self.device) if high_vram is None else bool(high_vram)
        self._high_vram = hv
        self.n_octaves = n_octaves if n_octaves is not None else (5 if hv else 4)
        self.n_scales = n_scales
        self.sigma0 = sigma0
        self.contrast_thresh = contrast_thresh
        self.edge_thresh = edge_thresh
        self.rootsift = rootsift
        self.as_uint8 = bool(as_uint8)
        self.dsp = dsp
        self.dsp_n_scales = dsp_n_scales
        self._dsp_scales_np = DSP_PRESETS[dsp_n_scales]
        self.fp16_pyramid = fp16_pyramid if fp16_pyramid is not None else (not hv)
        self.orientation = orientation
        self.descriptor = descriptor
        self.double_image = double_image
        self._lib = _lib.load()
        self._cfg = build_detect_config(self.n_octaves, n_scales, sigma0, contrast_thresh, edge_thresh, dsp,
                                        dsp_n_scales, self.fp16_pyramid, double_image, rootsift, hv)
        self._bufs = {}
        self._use_graphs = bool(graphs)
        self._phase_timings = None
        self._last_stats = None
        self._graphs = {}

    def autotune(self, H, W, path=None):
        """Measure (or load from the per-GPU JSON cache) the blur tile heights
        for detections of H x W images with this configuration and hand them
        to the library (pysift_b200.autotune); results do not change."""
        from . import autotune as _autotune
        return _autotune.autotune(self, H, W, path=path)

    # -- plumbing ---------------------------------------------------------
    def _buffers(self, H, W, slot=0):
        """Buffer set for one image size; distinct slots let detections of
        two images of the same size be in flight at once."""
        key = (H, W) if slot == 0 else (H, W, slot)
        b = self._bufs.get(key)
        if b is None:
            b = _Buffers(self._lib, self._cfg, H, W, self.device)
            self._bufs[key] = b
        return b

    def _launch(self, b, gray_dev, H, W, pitch, stream, stage_events=None):
        ev = None
        if stage_events is not None:
            if len(stage_events) != _lib.DETECT_STAGE_EVENTS:
                raise ValueError(f"stage_events needs {_lib.DETECT_STAGE_EVENTS} events")
            for e in stage_events:
                if not getattr(e, "_pysift_primed", False):
                    # torch creates the CUDA event on its first record() and only then
                    # reports timings; the library re-records the same handle.
                    e.record(torch.cuda.current_stream(self.device))
                    e._pysift_primed = True
            arr = (ctypes.c_void_p * _lib.DETECT_STAGE_EVENTS)(*[e.cuda_event for e in stage_events])
            ev = ctypes.cast(arr, ctypes.c_void_p)
        rc = self._lib.pysift_detect_and_compute(
            ctypes.byref(self._cfg), gray_dev, H, W, pitch, b.ws_ptr, b.ws_bytes,
            b.kpts.data_ptr(), b.resp.data_ptr(), b.octv.data_ptr(), b.desc.data_ptr(), b.max_out,
            b.stats.data_ptr(), ev, stream)
        _lib.check(rc, "pysift_detect_and_compute")

    def run_device(self, gray_t, stream=None, stage_events=None, slot=0):
        """Enqueue detection of a device uint8 (H, W) tensor on `stream`
        (default: the current stream).  Returns the buffer set holding the
        outputs; stats are read by the caller.  stage_events: optional list
        of 7 torch.cuda.Event recorded at the stage boundaries; slot selects
        an independent buffer set (for concurrent detections).  Unless the
        instance was built with graphs=False (or stage_events are asked for),
        the detection is a CUDA graph replay, captured on the first call for
        each image size, slot and configuration."""
        if gray_t.dtype != torch.uint8 or gray_t.dim() != 2:
            raise ValueError("expected a 2-D uint8 image")
        if gray_t.stride(1) != 1:
            gray_t = gray_t.contiguous()
        H, W = gray_t.shape
        b = self._buffers(H, W, slot)
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        if self._use_graphs and stage_events is None:
            self._run_graph(b, gray_t, H, W, slot, st)
        else:
            self._launch(b, gray_t.data_ptr(), H, W, gray_t.stride(0), st.cuda_stream, stage_events)
        return b

    def _run_graph(self, b, gray_t, H, W, slot, st):
        """Detection of one image as a CUDA graph replay.  The graph reads the
        buffer set's input image, so the image is copied there first (host
        uploads already land there); the first call for a size, slot and
        configuration runs eagerly and then captures the same launches."""
        if gray_t.data_ptr() != b.gray.data_ptr():
            with torch.cuda.stream(st):
                b.gray.copy_(gray_t, non_blocking=True)
        key = ("one", H, W, slot, bytes(self._cfg))
        ent = self._graphs.get(key)
        if ent is None:
            # the eager run goes on the capture stream, so the library's
            # per-stream side stream exists before the capture opens
            cap = self._capture_stream()
            cap.wait_stream(st)
            with torch.cuda.stream(cap):
                self._launch(b, b.gray.data_ptr(), H, W, W, cap.cuda_stream)
            st.wait_stream(cap)
            n0 = self._lib.pysift_launch_count()
            g = torch.cuda.CUDAGraph()
            capture_graph(g, cap, lambda: self._launch(b, b.gray.data_ptr(), H, W, W, cap.cuda_stream))
            n = self._lib.pysift_launch_count() - n0
            self._lib.pysift_count_launches(-n)  # captured, not run
            self._graphs[key] = (g, n)
            return
        g, n = ent
        with torch.cuda.stream(st):
            g.replay()
        self._lib.pysift_count_launches(n)

    def _capture_stream(self):
        if getattr(self, "_cap_stream", None) is None:
            self._cap_stream = torch.cuda.Stream(self.device)
        return self._cap_stream

    def _upload(self, gray, b):
        """Host numpy image -> pinned staging -> device (async on the current stream)."""
        b.gray_host.numpy()[...] = gray
        b.gray.copy_(b.gray_host, non_blocking=True)
        return b.gray

    # -- public API ---------------------------------------------------------
    def detectAndCompute(self, gray, mask=None, profile=False, gpu_output=False):
        """Detect keypoints and compute descriptors (pysift/core.py:2021-2172).

        gray: numpy uint8 (H, W) or a torch CUDA uint8 tensor.  Returns
        (list of cv2.KeyPoint, float32 (N,128) numpy) or, with gpu_output,
        torch CUDA tensors (N,4) [x, y, size, angle] and (N,128)."""
        del mask  # ignored, as in the reference
        if profile:
            torch.cuda.synchronize(self.device)
            t0 = time.perf_counter()
        with torch.cuda.device(self.device):
            if isinstance(gray, torch.Tensor):
                if not gray.is_cuda:
                    gray = gray.numpy()
            if isinstance(gray, np.ndarray):
                if gray.dtype != np.uint8 or gray.ndim != 2:
                    raise ValueError("gray must be a 2-D uint8 image")
                H, W = gray.shape
                b = self._buffers(H, W)
                g = self._upload(gray, b)
            else:
                g = gray
            b = self.run_device(g)
            b.stats_host.copy_(b.stats, non_blocking=True)
            torch.cuda.current_stream(self.device).synchronize()
            stats = b.stats_host.numpy().copy()
        self._last_stats = stats
        n = int(stats[_lib.STAT_N_KEYPOINTS])
        if profile:
            t1 = time.perf_counter()
            self._phase_timings = {'total_ms': (t1 - t0) * 1000.0}
        desc_dev = self._desc_u8(b.desc[:n]) if self.as_uint8 else b.desc[:n]
        if gpu_output:
            return b.kpts[:n].clone(), desc_dev.clone()
        kp = b.kpts[:n].cpu().numpy()
        resp = b.resp[:n].cpu().numpy()
        octv = b.octv[:n].cpu().numpy()
        desc = desc_dev.cpu().numpy()
        if n == 0:
            return [], np.zeros((0, 128), np.uint8 if self.as_uint8 else np.float32)
        return keypoints_from_rows(kp, resp, octv), desc

    def _desc_u8(self, desc):
        """OpenCV's uint8 form saturate(rint(512 v)) of float descriptors (device)."""
        out = torch.empty(desc.shape, dtype=torch.uint8, device=desc.device)
        _lib.check(self._lib.pysift_desc_to_u8(desc.data_ptr(), desc.shape[0], out.data_ptr(),
                                               torch.cuda.current_stream(desc.device).cuda_stream),
                   "pysift_desc_to_u8")
        return out

    # -- batched detection ----------------------------------------------------
    def detect_batch(self, images, n_streams=8, gpu_output=True, graph=False):
        """Detect and describe a list of grayscale uint8 images of any sizes in
        one call.  Images (numpy arrays or CUDA tensors) are dealt, largest
        first, to `n_streams` slots; each slot runs its images in order on its
        own CUDA stream with its own workspace (sized for its largest image),
        so detections of different images overlap on the GPU; every image has
        its own output buffers and the host waits once, after all of them.

        Returns a list of (kpts (N,4) [x, y, size, angle], desc (N,128)) per
        image, in input order: torch CUDA tensors with gpu_output, else numpy
        arrays.  n_streams=1 runs the same work back to back on one stream.

        graph=True replays the whole batch as one CUDA graph: the first call
        for a list of image shapes runs the batch once, then captures it
        (every stream's launches, forked from and joined back to one capture
        stream); later calls with the same shapes copy the images into the
        graph's input buffers and replay it.  Results are identical."""
        n = len(images)
        if n == 0:
            return []
        with torch.cuda.device(self.device):
            gray = []
            for img in images:
                if isinstance(img, torch.Tensor) and img.is_cuda:
                    t = img
                else:
                    a = np.ascontiguousarray(img)
                    if a.dtype != np.uint8 or a.ndim != 2:
                        raise ValueError("images must be 2-D uint8")
                    t = torch.from_numpy(a).to(self.device)
                if t.dtype != torch.uint8 or t.dim() != 2:
                    raise ValueError("images must be 2-D uint8")
                if t.stride(1) != 1:
                    t = t.contiguous()
                gray.append(t)
            if graph:
                return self._detect_batch_graph(gray, n_streams, gpu_output)
            self._enqueue_batch(gray, n_streams)
            torch.cuda.current_stream(self.device).synchronize()
            return self._collect_batch(n, gpu_output)

    def _enqueue_batch(self, gray, n_streams):
        """Enqueue the detection of every image of `gray` (device uint8
        tensors): images dealt largest first to the slot streams, forked from
        and joined back to the current stream; stats copied to pinned memory."""
        lib = self._lib
        n = len(gray)
        main = torch.cuda.current_stream(self.device)
        order = sorted(range(n), key=lambda i: -(gray[i].shape[0] * gray[i].shape[1]))
        ns = max(1, min(int(n_streams), n))
        slots = [order[s::ns] for s in range(ns)]
        if not hasattr(self, "_batch"):
            self._batch = {"streams": [], "ws": [], "outs": []}
        bt = self._batch
        while len(bt["streams"]) < ns:
            bt["streams"].append(torch.cuda.Stream(self.device))
            bt["ws"].append(None)
        max_out = int(lib.pysift_detect_max_keypoints(ctypes.byref(self._cfg)))
        while len(bt["outs"]) < n:
            bt["outs"].append(_BatchOutputs(max_out, self.device))
        for s, idxs in enumerate(slots):
            need = 0
            for i in idxs:
                H, W = gray[i].shape
                sz = ctypes.c_size_t(0)
                _lib.check(lib.pysift_detect_workspace_size(ctypes.byref(self._cfg), H, W, ctypes.byref(sz)),
                           "pysift_detect_workspace_size")
                need = max(need, int(sz.value))
            ws = bt["ws"][s]
            if ws is None or ws.numel() < need + 256:
                ws = torch.empty(need + 256, dtype=torch.uint8, device=self.device)
                bt["ws"][s] = ws
            st = bt["streams"][s]
            st.wait_stream(main)
            wptr = ws.data_ptr() + ((-ws.data_ptr()) % 256)
            with torch.cuda.stream(st):
                for i in idxs:
                    H, W = gray[i].shape
                    o = bt["outs"][i]
                    rc = lib.pysift_detect_and_compute(
                        ctypes.byref(self._cfg), gray[i].data_ptr(), H, W, gray[i].stride(0), wptr, need,
                        o.kpts.data_ptr(), o.resp.data_ptr(), o.octv.data_ptr(), o.desc.data_ptr(), max_out,
                        o.stats.data_ptr(), None, st.cuda_stream)
                    _lib.check(rc, "pysift_detect_and_compute")
                    o.stats_host.copy_(o.stats, non_blocking=True)
        for s in range(ns):
            main.wait_stream(bt["streams"][s])

    def _collect_batch(self, n, gpu_output):
        """The results of the last enqueued batch (the stream has finished)."""
        bt = self._batch
        out = []
        for i in range(n):
            o = bt["outs"][i]
            k = int(o.stats_host[_lib.STAT_N_KEYPOINTS])
            d = self._desc_u8(o.desc[:k]) if self.as_uint8 else o.desc[:k]
            if gpu_output:
                out.append((o.kpts[:k].clone(), d.clone()))
            else:
                out.append((o.kpts[:k].cpu().numpy(), d.cpu().numpy()))
        return out

    def _detect_batch_graph(self, gray, n_streams, gpu_output):
        key = (tuple(tuple(g.shape) for g in gray), int(n_streams))
        ent = self._graphs.get(key)
        main = torch.cuda.current_stream(self.device)
        if ent is None:
            # inputs live in buffers the graph reads; the first run (eager)
            # sizes the workspaces and outputs, the capture records the same
            # launches on those buffers
            inp = [torch.empty_like(g) for g in gray]
            for b, g in zip(inp, gray):
                b.copy_(g)
            self.detect_batch(inp, n_streams=n_streams, gpu_output=True)
            torch.cuda.synchronize(self.device)
            g_ = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g_):
                self._enqueue_batch(inp, n_streams)
            ent = (g_, inp)
            self._graphs[key] = ent
        g_, inp = ent
        for b, g in zip(inp, gray):
            b.copy_(g, non_blocking=True)
        g_.replay()
        main.synchronize()
        return self._collect_batch(len(gray), gpu_output)

    def detect_arrays(self, gray):
        """Host uint8 image in, host numpy arrays out: dict with x, y, size,
        angle, response, octave and desc (the reference's output rows,
        without building cv2.KeyPoint objects)."""
        with torch.cuda.device(self.device):
            H, W = gray.shape
            b = self._buffers(H, W)
            g = self._upload(gray, b)
            b = self.run_device(g)
            b.stats_host.copy_(b.stats, non_blocking=True)
            torch.cuda.current_stream(self.device).synchronize()
            stats = b.stats_host.numpy().copy()
            n = int(stats[_lib.STAT_N_KEYPOINTS])
            kp = b.kpts[:n].cpu().numpy()
            out = dict(x=kp[:, 0].copy(), y=kp[:, 1].copy(), size=kp[:, 2].copy(), angle=kp[:, 3].copy(),
                       response=b.resp[:n].cpu().numpy(), octave=b.octv[:n].cpu().numpy(),
                       desc=b.desc[:n].cpu().numpy())
        self._last_stats = stats
        return out

    @property
    def last_stats(self):
        """Counters of the last call (see include/pysift_b200.h PYSIFT_STAT_*)."""
        return self._last_stats
