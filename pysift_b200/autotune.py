"""Autotuner for the blur's tile height, cached per GPU in JSON.

The separable blur (k_blur, one launch per pyramid level) runs 64-column
tiles of 16, 32 or 40 rows.  The library's built-in rule picks the height
from the level size and the kernel's occupancy; this tuner measures all
three heights on the device for every (radius, level size class) a
detection of a given image size uses, keeps the fastest, hands the table to
the library (pysift_set_blur_tile_table) and stores it in
$PYSIFT_TUNE_CACHE (default ~/.cache/pysift_b200)/blur_tiles_<GPU>.json.
Results never depend on the table, only the time does.  The reference has
no counterpart (its blur launches have one shape, pysift/core.py:583-602).
"""
import ctypes
import json
import os

import numpy as np
import torch

from . import _lib

N_RADII = 17          # radius 0 .. 16
N_CLASSES = 16        # level size classes (floor(log2(pixels)) - 10)
ROWS = (16, 32, 40)   # the tile heights the library has


def cache_path(device=None):
    base = os.environ.get("PYSIFT_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "pysift_b200")
    name = torch.cuda.get_device_name(device).replace(" ", "_").replace("/", "_")
    return os.path.join(base, f"blur_tiles_{name}.json")


def pyramid_levels(sift, H, W):
    """(radius, level rows, level columns) of every blur a detection of an
    H x W image runs with this PySIFT configuration."""
    cfg = sift._cfg
    doubled = bool(cfg.double_image) and H * W < cfg.double_px_cap
    h, w = (2 * H, 2 * W) if doubled else (H, W)
    out = [(int(cfg.blur_radius[0 if doubled else 1]), h, w)]
    for _ in range(cfg.n_octaves):
        for s in range(cfg.n_scales + 2):
            out.append((int(cfg.blur_radius[2 + s]), h, w))
        h, w = (h + 1) // 2, (w + 1) // 2
    return out


def _time_blur(lib, R, h, w, rows, device, repeats):
    pitch = (w + 31) // 32 * 32
    src = torch.rand((h, pitch), dtype=torch.float32, device=device)
    dst = torch.empty_like(src)
    k = np.exp(-0.5 * (np.arange(-R, R + 1, dtype=np.float64) / max(R / 4.0, 0.5)) ** 2)
    k = np.ascontiguousarray(k / k.sum(), dtype=np.float32)
    st = torch.cuda.current_stream(device)
    _lib.check(lib.pysift_set_blur_tile_rows(rows), "pysift_set_blur_tile_rows")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    times = []
    for i in range(repeats + 3):
        ev[0].record(st)
        _lib.check(lib.pysift_gauss_blur(src.data_ptr(), pitch, dst.data_ptr(), pitch, h, w,
                                         k.ctypes.data_as(ctypes.c_void_p), R, st.cuda_stream), "pysift_gauss_blur")
        ev[1].record(st)
        ev[1].synchronize()
        if i >= 3:
            times.append(ev[0].elapsed_time(ev[1]))
    return float(np.median(times))


def tune(levels, device=None, repeats=15):
    """Measure every tile height for each (radius, h, w) of `levels`;
    returns {(radius, size class): rows} with the fastest height (the first
    on equal times)."""
    lib = _lib.load()
    device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    best = {}
    try:
        with torch.cuda.device(device):
            for R, h, w in sorted(set(levels)):
                if not 1 <= R < N_RADII:
                    continue
                key = (R, lib.pysift_blur_size_class(h, w))
                if key in best:
                    continue
                t = [(_time_blur(lib, R, h, w, rows, device, repeats), rows) for rows in ROWS]
                best[key] = min(t)[1]
    finally:
        lib.pysift_set_blur_tile_rows(0)
    return best


def to_table(best):
    table = np.zeros(N_RADII * N_CLASSES, np.int32)
    for (R, c), rows in best.items():
        table[R * N_CLASSES + c] = rows
    return table


def apply(best):
    """Hand the tuned heights to the library (later detections use them)."""
    table = to_table(best)
    _lib.check(_lib.load().pysift_set_blur_tile_table(table.ctypes.data_as(ctypes.c_void_p), table.size),
               "pysift_set_blur_tile_table")


def clear():
    _lib.check(_lib.load().pysift_set_blur_tile_table(None, 0), "pysift_set_blur_tile_table")


def save(best, path):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump({"blur_tile_rows": [[R, c, rows] for (R, c), rows in sorted(best.items())]}, f)


def load(path):
    with open(path) as f:
        d = json.load(f)
    return {(int(R), int(c)): int(rows) for R, c, rows in d["blur_tile_rows"]}


def autotune(sift, H, W, path=None, repeats=15):
    """Tile heights for detections of H x W images with this PySIFT: the
    cached ones when every (radius, size class) is in the cache file, else
    measured now and added to it; then applied.  Returns the table used."""
    path = path or cache_path(sift.device)
    levels = pyramid_levels(sift, H, W)
    lib = _lib.load()
    need = {(R, lib.pysift_blur_size_class(h, w)) for R, h, w in levels if 1 <= R < N_RADII}
    best = load(path) if os.path.exists(path) else {}
    if not need <= set(best):
        best.update(tune(levels, sift.device, repeats))
        save(best, path)
    apply(best)
    return best
