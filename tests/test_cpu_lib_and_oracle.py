"""CPU tests: the C-ABI library loads and exports what the header declares,
the host config mirrors the reference's host computations, and the oracle's
building blocks agree with their references (scipy zoom, libm functions)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    src = open(os.path.join(ROOT, "include", "pysift_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(pysift_[a-z0-9_]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_builds_and_exports_header_symbols():
    from pysift_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    names = _header_functions()
    assert len(names) >= 8
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/pysift_b200.h but not exported"


def test_binding_loads_and_struct_layout():
    from pysift_b200 import _lib
    lib = _lib.load()
    assert lib.pysift_detect_config_size() == ctypes.sizeof(_lib.DetectConfig)
    assert b"sm_100a" in lib.pysift_b200_version()
    for n in _header_functions():
        assert n in _lib.EXPORTS, f"{n} has no ctypes binding"


def test_workspace_size_and_errors():
    from pysift_b200 import _lib
    from pysift_b200.core import build_detect_config
    lib = _lib.load()
    cfg = build_detect_config(5, 3, 1.6, 0.04, 10.0, False, 3, False, True, True, True)
    sz = ctypes.c_size_t()
    assert lib.pysift_detect_workspace_size(ctypes.byref(cfg), 480, 640, ctypes.byref(sz)) == 0
    assert sz.value > 1280 * 960 * 6 * 4
    assert lib.pysift_detect_workspace_size(ctypes.byref(cfg), 0, 640, ctypes.byref(sz)) == _lib.ERR_INVALID_ARG
    assert b"positive" in lib.pysift_last_error()
    bad = build_detect_config(5, 3, 1.6, 0.04, 10.0, False, 3, False, True, True, True)
    bad.n_octaves = 9
    assert lib.pysift_detect_workspace_size(ctypes.byref(bad), 480, 640, ctypes.byref(sz)) == _lib.ERR_INVALID_ARG
    # argument checks run before any device work: NULL pointers are rejected on a CPU-only host
    rc = lib.pysift_detect_and_compute(ctypes.byref(cfg), None, 480, 640, 640, None, 0, None, None, None, None,
                                       32000, None, None, None)
    assert rc == _lib.ERR_INVALID_ARG


def test_config_tables_match_reference_host_math():
    from pysift_b200.core import build_detect_config, gaussian_weights
    cfg = build_detect_config(5, 3, 1.6, 0.04, 10.0, False, 3, False, True, True, True)
    # pysift/core.py:1283-1290: base blur sqrt(1.6^2 - 1), increments sqrt(s_i^2 - s_{i-1}^2)
    assert [cfg.blur_radius[i] for i in range(7)] == [5, 6, 5, 6, 8, 10, 12]
    w, r = gaussian_weights(float(np.sqrt(1.6 ** 2 - 1.0)), 4)
    assert np.array_equal(np.array(cfg.blur_weights[0][:2 * r + 1], np.float32), w)
    assert abs(float(np.sum(w)) - 1.0) < 1e-6
    assert [cfg.desc_ph[s] for s in (1, 2, 3)] == [21.0, 27.0, 34.0]
    assert np.float32(cfg.ori_sigma[3]) == np.float32(3.2)
    assert np.float32(cfg.edge_score) == np.float32(12.1)
    assert cfg.double_px_cap == 16_000_000
    low = build_detect_config(4, 3, 1.6, 0.04, 10.0, True, 5, True, True, True, False)
    assert low.double_px_cap == 4_194_304 and low.n_dsp == 5 and low.fp16_pyramid == 1


@pytest.mark.parametrize("shape", [(480, 640), (61, 37), (7, 9), (2, 3)])
def test_oracle_zoom_matches_scipy(shape, oracle_lib):
    import scipy.ndimage as nd
    rng = np.random.default_rng(sum(shape))
    img = (rng.random(shape) * 255).astype(np.uint8)
    base = img.astype(np.float32) / np.float32(255.0)
    ours = oracle_lib.zoom2x(base)
    ref = nd.zoom(base, 2.0, order=3)
    ulp = np.abs(ours.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1
    assert np.mean(ulp == 0) > 0.999


def _math_lib(oracle_lib):
    lib = oracle_lib.lib()
    for n in ("orc_test_expf", "orc_test_atan2f", "orc_test_sincosf", "orc_test_log2d"):
        getattr(lib, n).restype = None
    return lib


def test_oracle_elementary_functions_accuracy(oracle_lib):
    lib = _math_lib(oracle_lib)
    P = ctypes.c_void_p
    rng = np.random.default_rng(0)
    # exp on the ranges the SIFT weights use
    x = np.concatenate([-rng.random(20000) * 20, np.linspace(-10, 0, 1001)]).astype(np.float32)
    out = np.empty_like(x)
    lib.orc_test_expf(x.ctypes.data_as(P), out.ctypes.data_as(P), x.size)
    ref = np.exp(x.astype(np.float64))
    assert np.max(np.abs(out - ref) / ref) < 3e-7
    # atan2 over all quadrants and the zero cases the gradient produces
    y = (rng.standard_normal(20000) * rng.choice([1e-3, 1, 1e3], 20000)).astype(np.float32)
    xx = (rng.standard_normal(20000) * rng.choice([1e-3, 1, 1e3], 20000)).astype(np.float32)
    y[:4] = [0, 0, 1, -1]
    xx[:4] = [0, -1, 0, 0]
    out = np.empty_like(y)
    lib.orc_test_atan2f(y.ctypes.data_as(P), xx.ctypes.data_as(P), out.ctypes.data_as(P), y.size)
    ref = np.arctan2(y.astype(np.float64), xx.astype(np.float64))
    assert np.max(np.abs(out - ref)) < 1e-6
    assert out[0] == 0.0 and abs(out[1] - math.pi) < 1e-6
    # sin/cos on [0, 2 pi)
    a = (rng.random(20000) * 2 * math.pi).astype(np.float32)
    s = np.empty_like(a)
    c = np.empty_like(a)
    lib.orc_test_sincosf(a.ctypes.data_as(P), s.ctypes.data_as(P), c.ctypes.data_as(P), a.size)
    assert np.max(np.abs(s - np.sin(a.astype(np.float64)))) < 3e-7
    assert np.max(np.abs(c - np.cos(a.astype(np.float64)))) < 3e-7
    # log2 (double) on probabilities
    p = np.concatenate([rng.random(10000), 1.0 / np.arange(1, 5000)]).astype(np.float64)
    out = np.empty_like(p)
    lib.orc_test_log2d(p.ctypes.data_as(P), out.ctypes.data_as(P), p.size)
    assert np.max(np.abs(out - np.log2(p))) < 1e-14


def test_oracle_detect_runs_and_is_sorted(oracle_lib):
    from pysift_b200 import synthetic
    img = synthetic.scene(240, 320, seed=1)
    r = oracle_lib.OracleSIFT().detect_and_compute(img)
    n = len(r["x"])
    assert n > 50
    order = np.lexsort((r["y"], r["x"]))
    assert np.array_equal(order, np.arange(n))
    assert np.allclose(np.linalg.norm(r["desc"], axis=1), 1.0, atol=1e-5)


def test_fast_keypoint_and_dmatch_construction():
    """keypoints_from_rows / to_dmatches build the same cv2 objects as the
    reference's per-row constructors (pysift/core.py:2139-2142, 2929-2934)."""
    import cv2
    import torch
    from pysift_b200.core import keypoints_from_rows
    from pysift_b200.match import to_dmatches
    rng = np.random.default_rng(5)
    kp = (rng.random((300, 4)) * 500).astype(np.float32)
    resp = rng.random(300).astype(np.float32)
    octv = rng.integers(0, 5, 300).astype(np.int32)
    fast = keypoints_from_rows(kp, resp, octv)
    for j in (0, 17, 299):
        ref = cv2.KeyPoint(float(kp[j, 0]), float(kp[j, 1]), float(kp[j, 2]), float(kp[j, 3]), float(resp[j]),
                           int(octv[j]))
        k = fast[j]
        assert (k.pt, k.size, k.angle, k.response, k.octave) == (ref.pt, ref.size, ref.angle, ref.response,
                                                                   ref.octave)
    pairs = torch.tensor([[0, 5], [3, 1], [7, 2]], dtype=torch.int32)
    dist = torch.tensor([0.5, 0.25, 0.125], dtype=torch.float32)
    dm = to_dmatches(dict(pairs=pairs, dist=dist, count=torch.tensor([2], dtype=torch.int32)))
    assert [(d.queryIdx, d.trainIdx, d.distance, d.imgIdx) for d in dm] == [(0, 5, 0.5, -1), (3, 1, 0.25, -1)]
    assert to_dmatches(dict(pairs=pairs, dist=dist, count=torch.tensor([0], dtype=torch.int32))) == []


def test_as_uint8_requires_plain_sift():
    from pysift_b200 import PySIFT
    with pytest.raises(ValueError):
        PySIFT(as_uint8=True)


def test_product_never_imports_the_oracle():
    """The package is the product; the oracle is test infrastructure only.
    No module of pysift_b200 imports, loads or executes anything under
    oracle/, so a missing CUDA library can only fail, never fall back."""
    import ast
    import pathlib
    pkg = pathlib.Path(__file__).resolve().parent.parent / "pysift_b200"
    for py in sorted(pkg.rglob("*.py")):
        tree = ast.parse(py.read_text(), str(py))
        for node in ast.walk(tree):
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                names = [node.module or ""]
            else:
                continue
            assert not any(n == "oracle" or n.startswith("oracle.") for n in names), f"{py.name} imports the oracle"
        src = py.read_text()
        assert "liboracle" not in src and "oracle/" not in src, f"{py.name} names an oracle file"


@pytest.mark.parametrize("n_points,n_hyp", [(4, 1), (5, 155), (157, 156), (1000, 2048), (65537, 700)])
def test_ransac_samples_equal_torch_randint(n_points, n_hyp):
    """The reference draws its 4-point samples as torch.randint(0, N, (B, 4))
    from a CPU generator seeded with 42 (pysift/core.py:3011-3060).  The
    library's host stream (pysift_mt19937_u32) and the oracle's, reduced
    modulo N as the RANSAC kernels do, give the same indices; the lengths
    cross the 624-word MT19937 regeneration."""
    import torch
    from oracle import stitch_oracle as so
    from pysift_b200 import _lib
    lib = _lib.load()
    host = np.empty(4 * n_hyp, np.uint32)
    lib.pysift_mt19937_u32(42, host.ctypes.data_as(ctypes.c_void_p), host.size)
    assert np.array_equal(host, so.mt19937_u32(42, 4 * n_hyp))
    gen = torch.Generator(device="cpu")
    gen.manual_seed(42)
    want = torch.randint(0, n_points, (n_hyp, 4), generator=gen).numpy().ravel()
    assert np.array_equal((host % np.uint32(n_points)).astype(np.int64), want)
