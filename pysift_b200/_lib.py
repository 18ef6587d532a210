"""ctypes binding of libpysift_b200.so (declared in include/pysift_b200.h).

The library is loaded from the package directory; there is no fallback: a
missing or unloadable library raises immediately.
"""
import ctypes
import os

from . import build as _build

c_int32, c_int64, c_float, c_double = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_double
c_void_p, c_size_t = ctypes.c_void_p, ctypes.c_size_t

MAX_OCTAVES = 8
MAX_LEVELS = 8
MAX_RADIUS = 48
MAX_TAPS = 2 * MAX_RADIUS + 1

OK = 0
ERR_INVALID_ARG = -1
ERR_WORKSPACE = -2
ERR_CUDA = -3
ERR_UNSUPPORTED = -4
ERR_CAPACITY = -5

STAT_N_KEYPOINTS = 0
STAT_N_REFINED = 1
STAT_N_KEPT = 2
STAT_RETRIED = 3
STAT_CAPPED = 4
STAT_DOUBLED = 5
STAT_CAND_OVERFLOW = 6
STAT_CANDS = 8
STAT_REFINED_OCT = 16
STAT_THRESH_BITS = 24
STAT_COUNT = 32
DETECT_STAGE_EVENTS = 7


class DetectConfig(ctypes.Structure):
    """Mirror of pysift_detect_config."""
    _fields_ = [
        ("n_octaves", c_int32),
        ("n_scales", c_int32),
        ("sigma0", c_float),
        ("contrast_thresh", c_double),
        ("edge_score", c_float),
        ("double_image", c_int32),
        ("double_px_cap", c_int64),
        ("fp16_pyramid", c_int32),
        ("dsp", c_int32),
        ("n_dsp", c_int32),
        ("dsp_scales", c_float * 8),
        ("rootsift", c_int32),
        ("max_cands_per_octave", c_int32),
        ("keypoint_cap", c_int32),
        ("starvation_min", c_int32),
        ("border", c_int32),
        ("blur_radius", c_int32 * (2 + MAX_LEVELS)),
        ("blur_weights", (c_float * MAX_TAPS) * (2 + MAX_LEVELS)),
        ("ori_sigma", c_float * MAX_LEVELS),
        ("desc_ph", c_float * MAX_LEVELS),
        ("kp_size", ((c_float * MAX_LEVELS) * MAX_OCTAVES) * 2),
        ("output_limit", c_int32),
    ]


class PySiftError(RuntimeError):
    pass


_lib = None

EXPORTS = {
    # name: (restype, argtypes)
    "pysift_last_error": (ctypes.c_char_p, []),
    "pysift_b200_version": (ctypes.c_char_p, []),
    "pysift_launch_count": (c_int64, []),
    "pysift_count_launches": (None, [c_int64]),
    "pysift_host_copy": (ctypes.c_int, [c_void_p, c_void_p, c_size_t, c_int32]),
    "pysift_detect_config_size": (c_size_t, []),
    "pysift_detect_workspace_size": (ctypes.c_int, [c_void_p, c_int32, c_int32, ctypes.POINTER(c_size_t)]),
    "pysift_detect_max_keypoints": (c_int32, [c_void_p]),
    "pysift_detect_and_compute": (ctypes.c_int, [c_void_p, c_void_p, c_int32, c_int32, c_int64, c_void_p, c_size_t,
                                                 c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p,
                                                 c_void_p]),
    "pysift_detect_workspace_view": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32,
                                                    ctypes.POINTER(c_size_t), ctypes.POINTER(c_int32),
                                                    ctypes.POINTER(c_int32), ctypes.POINTER(c_int32)]),
    "pysift_gauss_blur": (ctypes.c_int, [c_void_p, c_int32, c_void_p, c_int32, c_int32, c_int32, c_void_p, c_int32,
                                         c_void_p]),
    "pysift_set_blur_tile_rows": (ctypes.c_int, [c_int32]),
    "pysift_blur_size_class": (ctypes.c_int, [c_int32, c_int32]),
    "pysift_set_blur_tile_table": (ctypes.c_int, [c_void_p, c_int32]),
    "pysift_zoom2x_u8": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int64, c_int32, c_void_p, c_void_p, c_int32,
                                        c_void_p]),
    "pysift_zoom2x_u8_noalloc": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int64, c_int32, c_void_p, c_int32,
                                                c_void_p]),
}
ZOOM2X_NOALLOC_MAX_PIXELS = 1 << 20

EXPORTS.update({
    "pysift_match_workspace_size": (ctypes.c_int, [c_int32, c_int32, c_int32, c_int32, ctypes.POINTER(c_size_t)]),
    "pysift_match_fp16": (ctypes.c_int, [c_void_p, c_int32, c_void_p, c_int32, c_int32, c_float, c_void_p, c_size_t,
                                         c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                         c_void_p]),
    "pysift_match_fp16_recheck_counts": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p]),
    "pysift_match_u8_exact": (ctypes.c_int, [c_void_p, c_int32, c_void_p, c_int32, c_int32, c_float, c_void_p,
                                             c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                             c_void_p, c_void_p]),
    "pysift_desc_f32_forward": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_int32, c_int32,
                                               c_void_p, c_void_p, c_void_p]),
    "pysift_desc_f32_backward": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_int32, c_int32,
                                                c_void_p, c_void_p, c_void_p, c_void_p]),
    "pysift_blur_adjoint": (ctypes.c_int, [c_void_p, c_int32, c_void_p, c_int32, c_void_p, c_int32, c_int32, c_int32,
                                           c_void_p, c_int32, c_int32, c_void_p]),
    "pysift_warp_f32_forward": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_int32, c_int32,
                                               c_int32, c_int32, c_void_p, c_double, c_double, c_int32, c_int32,
                                               c_void_p, c_void_p]),
    "pysift_warp_f32_backward": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_int32, c_int32,
                                                c_int32, c_int32, c_void_p, c_double, c_double, c_int32, c_int32,
                                                c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "pysift_match_u8_split_fp8": (ctypes.c_int, [c_void_p, c_int32, c_void_p, c_int32, c_int32, c_float, c_void_p,
                                                 c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                                 c_void_p, c_void_p, c_void_p]),
})


def lib_path():
    return _build.LIB_PATH


def load():
    """Load the shared library (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not os.path.exists(path):
        raise PySiftError(
            f"{path} is missing: build the CUDA library first (python -m pysift_b200.build)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.pysift_detect_config_size() != ctypes.sizeof(DetectConfig):
        raise PySiftError("pysift_detect_config layout mismatch between Python and the library")
    _lib = lib
    return lib


def check(rc, what):
    if rc != OK:
        msg = load().pysift_last_error().decode(errors="replace")
        if rc == ERR_INVALID_ARG:
            raise ValueError(f"{what}: {msg}")
        raise PySiftError(f"{what} failed ({rc}): {msg}")

EXPORTS.update({
    "pysift_bgr2gray": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int64, c_void_p, c_int32, c_void_p]),
    "pysift_desc_to_u8": (ctypes.c_int, [c_void_p, c_int64, c_void_p, c_void_p]),
    "pysift_clahe_lut_bytes": (ctypes.c_int, [c_int32, c_int32, ctypes.POINTER(c_size_t)]),
    "pysift_clahe": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_double, c_int32, c_int32, c_void_p,
                                    c_void_p, c_int32, c_void_p]),
    "pysift_topk_by_response": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p]),
    "pysift_gather_points": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p]),
    "pysift_l2_normalize_rows": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_void_p, c_void_p]),
    "pysift_pca_workspace_size": (ctypes.c_int, [c_int32, c_int32, ctypes.POINTER(c_size_t)]),
    "pysift_pca_basis_workspace_size": (ctypes.c_int, [c_int32, ctypes.POINTER(c_size_t)]),
    "pysift_pca_basis": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p]),
    "pysift_pca_stats": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_void_p, c_size_t, c_void_p, c_void_p,
                                        c_void_p]),
    "pysift_pca_project_f16": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_int32, c_void_p,
                                              c_void_p]),
    "pysift_to_f16": (ctypes.c_int, [c_void_p, c_int64, c_void_p, c_void_p]),
    "pysift_mt19937_u32": (None, [ctypes.c_uint32, c_void_p, c_int64]),
    "pysift_ransac_workspace_size": (ctypes.c_int, [c_int32, c_int32, ctypes.POINTER(c_size_t)]),
    "pysift_ransac": (ctypes.c_int, [c_void_p, c_void_p, c_int32, c_void_p, c_int32, c_double, c_double, c_int32,
                                     c_int32, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p]),
    "pysift_ransac_count": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_int32, c_double,
                                           c_double, c_int32, c_int32, c_void_p, c_size_t, c_void_p, c_void_p,
                                           c_void_p, c_void_p]),
    "pysift_dlt_homography": (ctypes.c_int, [c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p]),
    "pysift_warp_feather": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_int32, c_int32, c_int32,
                                           c_int32, c_int32, c_void_p, c_float, c_float, c_int32, c_int32, c_int32,
                                           c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                           c_void_p, c_void_p]),
    "pysift_pca_project_f32": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_int32, c_void_p,
                                              c_void_p]),
    "pysift_quantize_i8_rows": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p]),
    "pysift_match_i8": (ctypes.c_int, [c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_int32, c_int32, c_float,
                                       c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p]),
    "pysift_place_image": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32,
                                          c_void_p, c_void_p, c_void_p]),
    "pysift_blend_workspace_size": (ctypes.c_int, [c_int32, c_int32, c_int32, c_void_p]),
    "pysift_blend_multiband": (ctypes.c_int, [c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_int32,
                                              c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p,
                                              c_void_p, c_void_p, c_void_p, c_void_p]),
    "pysift_mask_extents": (ctypes.c_int, [c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                                           c_void_p]),
    "pysift_autocrop_box": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p]),
    "pysift_copy2d": (ctypes.c_int, [c_void_p, c_size_t, c_void_p, c_size_t, c_size_t, c_size_t, c_void_p]),
})
