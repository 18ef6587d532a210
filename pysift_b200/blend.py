"""The reference's two-image composition on the device: gain compensation,
dynamic-programming seam and Laplacian (multi-band) blend
(GPUPyStitch._blend_pair, pysift/core.py:3686-3714; _find_seam 3386-3472;
_multiband_blend 3495-3553; the paste of _stitch_pair 3806-3809) as one
C-ABI call, pysift_blend_multiband, with no host synchronisation.

Arithmetic: float32 images; gaussian_filter(sigma=1), sobel and
zoom(order=1) with scipy.ndimage's float64 line sums (the algorithms
cupyx.scipy.ndimage implements); the seam DP in float64 with numpy's
first-minimum tie order.  Two steps take a canonical form: the overlap means
of the gain are exact (the reference takes float32 pairwise means), and the
sigma-3 seam-mask blur is the separable 25-tap filter of :func:`seam_kernel`
with reflect-101 borders and float64 sums (the reference calls
cv2.GaussianBlur).
"""
import numpy as np
import torch

from . import _lib


def seam_kernel(sigma=3.0, taps=25):
    """float32 taps of the seam-mask blur: exp(-x^2 / (2 sigma^2)) normalised
    (the kernel cv2.GaussianBlur(sigmaX=3) builds: 25 taps for sigma 3)."""
    x = np.arange(taps, dtype=np.float64) - (taps - 1) / 2.0
    t = np.exp((-0.5 / (sigma * sigma)) * (x * x))
    return (t / t.sum()).astype(np.float32)


def gauss_weights(sigma=1.0, truncate=4.0):
    """float64 taps of scipy.ndimage.gaussian_filter1d(sigma) (radius
    int(truncate * sigma + 0.5))."""
    r = int(truncate * sigma + 0.5)
    x = np.arange(-r, r + 1)
    p = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    return p / p.sum()


_SEAM_K = seam_kernel()
_GAUSS_W = np.ascontiguousarray(gauss_weights(), dtype=np.float64)


def workspace_bytes(cw, ch, n_levels=6):
    lib = _lib.load()
    import ctypes
    n = ctypes.c_size_t()
    _lib.check(lib.pysift_blend_workspace_size(int(cw), int(ch), int(n_levels), ctypes.byref(n)),
               "pysift_blend_workspace_size")
    return n.value


def place_image(img, cw, ch, iox, ioy, canvas=None, mask=None, stream=None):
    """Image 2 (h, w, 3 uint8 on the device) pasted on a zero canvas at
    (iox, ioy) (pysift/core.py:3794-3800); returns (canvas, mask)."""
    lib = _lib.load()
    dev = img.device
    if canvas is None:
        canvas = torch.empty((ch, cw, 3), dtype=torch.uint8, device=dev)
    if mask is None:
        mask = torch.empty((ch, cw), dtype=torch.uint8, device=dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    h, w = img.shape[:2]
    _lib.check(lib.pysift_place_image(img.data_ptr(), h, w, img.stride(0), cw, ch, int(iox), int(ioy),
                                      canvas.data_ptr(), mask.data_ptr(), st), "pysift_place_image")
    return canvas, mask


def blend_multiband(image1, mask1, canvas2, mask2, n_levels=6, workspace=None, pano=None, both=None,
                    seam_rmse=None, blended=None, want_pano=True, stream=None, color_match="gain"):
    """_blend_pair + paste.  image1: (ch, cw, 3) uint8 (a warped image) or
    float32 (an earlier blend's unclipped result); canvas2: (ch, cw, 3)
    uint8; masks (ch, cw) uint8 / bool; all on the device.  Returns (pano
    uint8 (ch, cw, 3) or None, both uint8 (ch, cw), seam_rmse float64 (1,),
    blended float32 (ch, cw, 3) or None), enqueued on the current stream;
    pass a `blended` tensor to get the unclipped blend.  color_match 'hist'
    matches histograms (_hist_match), anything else applies the gain, as
    pysift/core.py:3694-3698 does."""
    lib = _lib.load()
    ch, cw = mask1.shape
    dev = mask1.device
    f32 = image1.dtype == torch.float32
    if image1.shape != (ch, cw, 3) or image1.dtype not in (torch.uint8, torch.float32) or \
            not image1.is_contiguous() or image1.device != dev:
        raise ValueError("image1 must be a contiguous (ch, cw, 3) uint8 or float32 tensor on the masks' device")
    if canvas2.shape != (ch, cw, 3) or canvas2.dtype != torch.uint8 or not canvas2.is_contiguous() or \
            canvas2.device != dev:
        raise ValueError("canvas2 must be a contiguous (ch, cw, 3) uint8 tensor on the masks' device")
    m1 = mask1.view(torch.uint8) if mask1.dtype == torch.bool else mask1
    m2 = mask2.view(torch.uint8) if mask2.dtype == torch.bool else mask2
    if m1.dtype != torch.uint8 or m2.shape != (ch, cw) or not (m1.is_contiguous() and m2.is_contiguous()):
        raise ValueError("masks must be contiguous (ch, cw) uint8 or bool")
    need = workspace_bytes(cw, ch, n_levels)
    if workspace is None or workspace.numel() < need + 256:
        workspace = torch.empty(need + 256, dtype=torch.uint8, device=dev)
    wp = workspace.data_ptr() + ((-workspace.data_ptr()) % 256)
    if pano is None and want_pano:
        pano = torch.empty((ch, cw, 3), dtype=torch.uint8, device=dev)
    if both is None:
        both = torch.empty((ch, cw), dtype=torch.uint8, device=dev)
    if seam_rmse is None:
        seam_rmse = torch.empty(1, dtype=torch.float64, device=dev)
    if pano is None and blended is None:
        raise ValueError("nothing to compute: want_pano=False and no blended tensor")
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    _lib.check(lib.pysift_blend_multiband(image1.data_ptr(), 1 if f32 else 0, m1.data_ptr(), canvas2.data_ptr(),
                                          m2.data_ptr(), cw, ch, int(n_levels), 1 if color_match == "hist" else 0,
                                          _SEAM_K.ctypes.data,
                                          _GAUSS_W.ctypes.data, wp, need, pano.data_ptr() if pano is not None else None,
                                          both.data_ptr(), blended.data_ptr() if blended is not None else None,
                                          seam_rmse.data_ptr(), st),
               "pysift_blend_multiband")
    return pano, both, seam_rmse, blended


def mask_extents(mask, out=None, stream=None):
    """Per-row / per-column first and last set pixel of a (ch, cw) uint8 mask
    on the device: int32 (2 ch + 2 cw,) = row_lo, row_hi, col_lo, col_hi."""
    lib = _lib.load()
    ch, cw = mask.shape
    if out is None:
        out = torch.empty(2 * ch + 2 * cw, dtype=torch.int32, device=mask.device)
    st = stream if stream is not None else torch.cuda.current_stream(mask.device).cuda_stream
    _lib.check(lib.pysift_mask_extents(mask.data_ptr(), cw, ch, out.data_ptr(), out[ch:].data_ptr(),
                                       out[2 * ch:].data_ptr(), out[2 * ch + cw:].data_ptr(), st),
               "pysift_mask_extents")
    return out
