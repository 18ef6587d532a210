"""GPU parity of the stitch-path kernels (gray, CLAHE, top-k, matcher prep,
RANSAC, DLT, warp + feather) and of the whole two-image stitch."""
import ctypes

import numpy as np
import pytest

from pysift_b200 import synthetic

pytestmark = pytest.mark.gpu


def _lib():
    from pysift_b200 import _lib
    return _lib, _lib.load()


def _st():
    import torch
    return torch.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("shape", [(960, 1280), (481, 643), (100, 77), (9, 13), (240, 2100), (243, 2096)])
def test_gray_and_clahe_match_cv2(shape):
    import cv2
    import torch
    L, lib = _lib()
    H, W = shape
    bgr = np.stack([synthetic.scene(H, W, seed=s) for s in range(3)], -1)
    g = torch.from_numpy(bgr).cuda()
    gray = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    assert lib.pysift_bgr2gray(g.data_ptr(), H, W, 3 * W, gray.data_ptr(), W, _st()) == 0
    ref = cv2.cvtColor(bgr, cv2.COLOR_BGR2GRAY)
    assert np.array_equal(gray.cpu().numpy(), ref)
    lut = torch.empty(64 * 256, dtype=torch.uint8, device="cuda")
    out = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    assert lib.pysift_clahe(gray.data_ptr(), H, W, W, 2.0, 8, 8, lut.data_ptr(), out.data_ptr(), W, _st()) == 0
    ref_c = cv2.createCLAHE(clipLimit=2.0, tileGridSize=(8, 8)).apply(ref)
    assert np.array_equal(out.cpu().numpy(), ref_c)


def test_topk_by_response_is_stable_descending():
    import torch
    L, lib = _lib()
    rng = np.random.default_rng(0)
    resp = rng.integers(0, 50, size=20000).astype(np.float32)  # many ties
    r = torch.from_numpy(resp).cuda()
    rank = torch.empty(20000, dtype=torch.int32, device="cuda")
    idx = torch.empty(8000, dtype=torch.int32, device="cuda")
    assert lib.pysift_topk_by_response(r.data_ptr(), 20000, 8000, rank.data_ptr(), idx.data_ptr(), _st()) == 0
    ref = np.array(sorted(range(20000), key=lambda i: -float(resp[i])))[:8000]
    assert np.array_equal(idx.cpu().numpy(), ref)


def test_matcher_preparation_bit_exact():
    import torch
    from oracle import stitch_oracle as so
    L, lib = _lib()
    rng = np.random.default_rng(1)
    d = np.abs(rng.standard_normal((3000, 128))).astype(np.float32)
    x = torch.from_numpy(d).cuda()
    out = torch.empty_like(x)
    assert lib.pysift_l2_normalize_rows(x.data_ptr(), 3000, 128, out.data_ptr(), _st()) == 0
    ref = so.l2_normalize(d)
    assert np.array_equal(out.cpu().numpy(), ref)
    mean = torch.empty(128, dtype=torch.float32, device="cuda")
    cov = torch.empty((128, 128), dtype=torch.float64, device="cuda")
    sz = ctypes.c_size_t()
    assert lib.pysift_pca_workspace_size(3000, 128, ctypes.byref(sz)) == 0
    ws = torch.empty(sz.value, dtype=torch.uint8, device="cuda")
    assert lib.pysift_pca_stats(out.data_ptr(), 3000, 128, ws.data_ptr(), ws.numel(), mean.data_ptr(),
                                cov.data_ptr(), _st()) == 0
    rmean, rcov = so.pca_stats(ref)
    assert np.array_equal(mean.cpu().numpy(), rmean)
    assert np.array_equal(cov.cpu().numpy(), rcov)
    # the basis: the device Jacobi equals the oracle's bit for bit
    proj = so.pca_basis(rcov, 64)
    pj = torch.empty((128, 64), dtype=torch.float32, device="cuda")
    assert lib.pysift_pca_basis_workspace_size(128, ctypes.byref(sz)) == 0
    wsb = torch.empty(sz.value, dtype=torch.uint8, device="cuda")
    sweeps = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.pysift_pca_basis(cov.data_ptr(), 128, 64, wsb.data_ptr(), wsb.numel(), pj.data_ptr(),
                                sweeps.data_ptr(), _st()) == 0
    assert np.array_equal(pj.cpu().numpy(), proj)
    assert so.pca_basis(rcov, 64, return_sweeps=True)[1] == int(sweeps.item())
    o16 = torch.empty((3000, 64), dtype=torch.float16, device="cuda")
    assert lib.pysift_pca_project_f16(out.data_ptr(), 3000, 128, mean.data_ptr(), pj.data_ptr(), 64, o16.data_ptr(),
                                      _st()) == 0
    rp = so.pca_project(ref, rmean, proj).astype(np.float16)
    assert np.array_equal(o16.cpu().numpy(), rp)


def _correspondences(seed, n=1500, outliers=0.3):
    rng = np.random.default_rng(seed)
    Ht = synthetic.random_homography(rng, 1280, 960)
    p1 = np.stack([rng.uniform(0, 1280, n), rng.uniform(0, 960, n)], 1)
    ph = np.hstack([p1, np.ones((n, 1))]) @ Ht.T
    p2 = ph[:, :2] / ph[:, 2:3] + rng.normal(0, 0.7, (n, 2))
    k = int(outliers * n)
    p2[:k] = np.stack([rng.uniform(-500, 1500, k), rng.uniform(-200, 1100, k)], 1)
    p1 = p1.astype(np.float32).astype(np.float64)
    p2 = p2.astype(np.float32).astype(np.float64)
    return p1, p2, Ht


@pytest.mark.parametrize("seed,magsac", [(0, True), (1, True), (2, False)])
def test_ransac_bit_exact(seed, magsac):
    import torch
    from oracle import stitch_oracle as so
    L, lib = _lib()
    p1, p2, Ht = _correspondences(seed)
    n, n_hyp = len(p1), 2048
    rnd = so.mt19937_u32(42, 4 * n_hyp)
    host = np.empty(4 * n_hyp, np.uint32)
    lib.pysift_mt19937_u32(42, host.ctypes.data_as(ctypes.c_void_p), host.size)
    assert np.array_equal(host, rnd)
    gen = torch.Generator(device="cpu")
    gen.manual_seed(42)
    ti = torch.randint(0, n, (n_hyp, 4), generator=gen).numpy().ravel()
    assert np.array_equal(ti, (rnd % n).astype(np.int64))
    sz = ctypes.c_size_t()
    lib.pysift_ransac_workspace_size(n, n_hyp, ctypes.byref(sz))
    ws = torch.empty(sz.value + 256, dtype=torch.uint8, device="cuda")
    off = (-ws.data_ptr()) % 256
    d1, d2 = torch.from_numpy(p1).cuda(), torch.from_numpy(p2).cuda()
    r = torch.from_numpy(rnd).cuda()
    H = torch.empty(9, dtype=torch.float64, device="cuda")
    mask = torch.empty(n, dtype=torch.uint8, device="cuda")
    info = torch.empty(3, dtype=torch.int32, device="cuda")
    rc = lib.pysift_ransac(d1.data_ptr(), d2.data_ptr(), n, r.data_ptr(), n_hyp, 4.0, 4.0, 1 if magsac else 0, 10,
                           ws.data_ptr() + off, sz.value, H.data_ptr(), mask.data_ptr(), info.data_ptr(), _st())
    assert rc == 0
    rH, rmask, rinfo, _ = so.ransac(p1, p2, n_hyp, 4.0, 4.0, magsac)
    assert np.array_equal(info.cpu().numpy(), rinfo)
    assert np.array_equal(mask.cpu().numpy().astype(bool), rmask)
    assert np.array_equal(H.cpu().numpy().reshape(3, 3), rH)
    # and it found the true geometry
    assert rinfo[0] > 0.6 * n
    Hn = rH / rH[2, 2]
    assert np.allclose(Hn, Ht / Ht[2, 2], rtol=5e-3, atol=5e-3 * np.abs(Ht).max())


def test_dlt_matches_oracle_and_svd():
    import torch
    from oracle import stitch_oracle as so
    L, lib = _lib()
    p1, p2, Ht = _correspondences(5, n=400, outliers=0.0)
    d1, d2 = torch.from_numpy(p1).cuda(), torch.from_numpy(p2).cuda()
    idx = torch.empty(400, dtype=torch.int32, device="cuda")
    H = torch.empty(9, dtype=torch.float64, device="cuda")
    assert lib.pysift_dlt_homography(d1.data_ptr(), d2.data_ptr(), 400, idx.data_ptr(), H.data_ptr(), _st()) == 0
    Hg = H.cpu().numpy().reshape(3, 3)
    assert np.array_equal(Hg, so.dlt(p1, p2))
    # the reference's SVD formulation (pysift/core.py:2959-2981) in float64
    def norm(p):
        c = p.mean(0); md = np.sqrt(((p - c) ** 2).sum(1)).mean(); s = np.sqrt(2) / (md + 1e-10)
        T = np.array([[s, 0, -s * c[0]], [0, s, -s * c[1]], [0, 0, 1]])
        return (T @ np.hstack([p, np.ones((len(p), 1))]).T).T[:, :2], T
    a, T1 = norm(p1); b, T2 = norm(p2)
    A = np.zeros((800, 9))
    for i in range(400):
        A[2 * i] = [-a[i, 0], -a[i, 1], -1, 0, 0, 0, b[i, 0] * a[i, 0], b[i, 0] * a[i, 1], b[i, 0]]
        A[2 * i + 1] = [0, 0, 0, -a[i, 0], -a[i, 1], -1, b[i, 1] * a[i, 0], b[i, 1] * a[i, 1], b[i, 1]]
    Hs = np.linalg.inv(T2) @ np.linalg.svd(A)[2][-1].reshape(3, 3) @ T1
    Hs /= Hs[2, 2]
    assert np.max(np.abs(Hg - Hs) / np.maximum(np.abs(Hs), 1e-9)) < 1e-6


def test_warp_feather_bit_exact_and_grid_sample():
    import torch
    import torch.nn.functional as F
    from oracle import stitch_oracle as so
    L, lib = _lib()
    img1, img2, Ht = synthetic.stitch_pair(240, 320, seed=3)
    Hs = np.linalg.inv(Ht)  # maps view-1 to view-2: use the true homography image1 -> image2 frame
    H = Ht
    cw, ch, ox, oy = so.canvas_size(img1.shape, img2.shape, H)
    hinv = np.linalg.inv(H).astype(np.float32)
    iox, ioy = int(round(ox)), int(round(oy))
    g1, g2 = torch.from_numpy(img1).cuda(), torch.from_numpy(img2).cuda()
    out = torch.empty((ch, cw, 3), dtype=torch.uint8, device="cuda")
    warped = torch.empty_like(out)
    m1 = torch.empty((ch, cw), dtype=torch.uint8, device="cuda")
    m2 = torch.empty_like(m1)
    hb = (ctypes.c_float * 9)(*[float(v) for v in hinv.ravel()])
    rc = lib.pysift_warp_feather(g1.data_ptr(), 240, 320, 960, g2.data_ptr(), 240, 320, 960, cw, ch,
                                 ctypes.cast(hb, ctypes.c_void_p), float(np.float32(ox)), float(np.float32(oy)), iox,
                                 ioy, 1, out.data_ptr(), warped.data_ptr(), m1.data_ptr(), m2.data_ptr(), None, None,
                                 None, None, _st())
    assert rc == 0
    r_out, r_warp, r_m1, r_m2 = so.warp_feather(img1, img2, hinv, cw, ch, ox, oy, iox, ioy)
    assert np.array_equal(out.cpu().numpy(), r_out)
    assert np.array_equal(warped.cpu().numpy(), r_warp)
    assert np.array_equal(m1.cpu().numpy().astype(bool), r_m1)
    assert np.array_equal(m2.cpu().numpy().astype(bool), r_m2)
    # the bilinear part equals torch's grid_sample on the same grid (the reference's call)
    u = torch.arange(cw, dtype=torch.float32, device="cuda")
    v = torch.arange(ch, dtype=torch.float32, device="cuda")
    uu, vv = torch.meshgrid(u, v, indexing="xy")
    X, Y = uu - float(np.float32(ox)), vv - float(np.float32(oy))
    hi = torch.from_numpy(hinv).cuda()
    s0 = hi[0, 0] * X + hi[0, 1] * Y + hi[0, 2]
    s1 = hi[1, 0] * X + hi[1, 1] * Y + hi[1, 2]
    s2 = hi[2, 0] * X + hi[2, 1] * Y + hi[2, 2]
    den = s2.clamp(min=1e-10)
    sxn = (2.0 * (s0 / den) / (320 - 1)) - 1.0
    syn = (2.0 * (s1 / den) / (240 - 1)) - 1.0
    grid = torch.stack([sxn, syn], -1).reshape(1, ch, cw, 2)
    it = g1.float().permute(2, 0, 1).unsqueeze(0)
    gs = F.grid_sample(it, grid, mode="bilinear", padding_mode="zeros", align_corners=True)
    ref_w = gs.squeeze(0).permute(1, 2, 0).cpu().numpy().clip(0, 255).astype(np.uint8)
    # (the cross-check with torch's kernel allows last-bit differences of its
    # accumulation at uint8 truncation boundaries)
    wv = warped.cpu().numpy()
    assert np.mean(ref_w == wv) > 0.999
    assert np.abs(ref_w.astype(int) - wv.astype(int)).max() <= 1


def _assert_stitch_equals_oracle(st, pano, orc):
    """Everything the two-image stitch produces equals the oracle: keypoint
    counts, the mutual pairs, RANSAC's inlier mask and homography, the canvas
    geometry, the composed canvas before the crop, and the crop."""
    m = st.last_metrics
    assert m["kp1"] == orc["n1"] and m["kp2"] == orc["n2"]
    assert np.array_equal(st._last["pairs"].cpu().numpy(), orc["pairs"])
    assert np.array_equal(st._last["mask"].cpu().numpy().astype(bool), orc["mask"])
    Hg = st._last["H"]
    rel = np.max(np.abs(Hg - orc["H"]) / np.maximum(np.abs(orc["H"]), 1e-300))
    assert rel < 1e-6, rel
    assert np.array_equal(Hg, orc["H"])
    c = st._last_compose
    assert (c["canvas_w"], c["canvas_h"]) == orc["canvas_size"]
    assert np.array_equal(c["out"].cpu().numpy(), orc["canvas"])
    assert pano.shape == orc["pano"].shape and np.array_equal(pano, orc["pano"])


@pytest.mark.parametrize("H,W,blend", [(480, 640, "feather"), (482, 640, "feather"), (480, 640, "multiband")])
def test_stitch_pair_end_to_end(H, W, blend):
    """The whole pair against the oracle; 482 x 640 has one side that does
    not divide by the CLAHE tile count (cv2 then extends both sides)."""
    from oracle import stitch_oracle as so
    from pysift_b200.stitch import GPUPyStitch
    img1, img2, Ht = synthetic.stitch_pair(H, W, seed=1)
    st = GPUPyStitch(ransac_iters=2048, inlier_thresh=4.0, save_output=False, verbose=False, blend=blend)
    pano = st.stitch(img1, img2)
    orc = so.OracleStitch(ransac_iters=2048, inlier_thresh=4.0, blend=blend).stitch(img1, img2)
    _assert_stitch_equals_oracle(st, pano, orc)
    Hg = st._last["H"]
    Ht_n = Ht / Ht[2, 2]
    assert np.allclose(Hg / Hg[2, 2], Ht_n, rtol=2e-2, atol=2e-2 * np.abs(Ht_n).max())


def test_stitch_bench_pair_end_to_end():
    """The benchmarked pair: 1280 x 960 BGR views of the seed-0 scene,
    GPUPyStitch(ransac_iters=2048, inlier_thresh=4.0) with its default
    multiband composition, against the oracle in every output."""
    from oracle import stitch_oracle as so
    from pysift_b200.stitch import GPUPyStitch
    img1, img2, _ = synthetic.stitch_pair(960, 1280, seed=0)
    st = GPUPyStitch(ransac_iters=2048, inlier_thresh=4.0, save_output=False, verbose=False)
    pano = st.stitch(img1, img2)
    orc = so.OracleStitch(ransac_iters=2048, inlier_thresh=4.0).stitch(img1, img2)
    _assert_stitch_equals_oracle(st, pano, orc)
    assert st.last_metrics["matches"] > 500 and st.last_metrics["inliers"] > 500


def test_stitch_pair_of_different_sizes():
    """Views of different sizes (the second cropped at its bottom and right
    edges, which keeps the true homography): every output against the oracle."""
    from oracle import stitch_oracle as so
    from pysift_b200.stitch import GPUPyStitch
    img1, img2, Ht = synthetic.stitch_pair(480, 640, seed=2)
    img2 = np.ascontiguousarray(img2[:473, :629])
    st = GPUPyStitch(ransac_iters=2048, inlier_thresh=4.0, save_output=False, verbose=False, blend="feather")
    pano = st.stitch(img1, img2)
    orc = so.OracleStitch(ransac_iters=2048, inlier_thresh=4.0, blend="feather").stitch(img1, img2)
    _assert_stitch_equals_oracle(st, pano, orc)


def test_stitch_batch_matches_sequential_stitch():
    """stitch_batch returns, pair for pair, the panorama that sequential
    stitch() calls on an instance in the same state return."""
    from pysift_b200.stitch import GPUPyStitch
    pairs = [synthetic.stitch_pair_fast(h, w, seed=50 + i)[:2] for i, (h, w) in
             enumerate([(480, 640), (600, 800), (500, 700)])]
    seq = GPUPyStitch(ransac_iters=512, inlier_thresh=4.0, save_output=False)
    ref = [seq.stitch(a, b) for a, b in pairs]
    bat = GPUPyStitch(ransac_iters=512, inlier_thresh=4.0, save_output=False)
    for n_streams in (4, 1):
        got = bat.stitch_batch(pairs, n_streams=n_streams)
        assert len(got) == len(pairs)
        for r, g in zip(ref, got):
            assert r.shape == g.shape and np.array_equal(r, g)


def test_pre_and_post_processing_options(tmp_path, monkeypatch):
    """max_dimension / denoise / sharpen preprocess the inputs with the
    reference's OpenCV calls (pysift/core.py:2486-2514): the stitch equals one
    of the preprocessed images; output_max_dim / post_sharpen change only the
    saved file (pysift/core.py:4054-4092)."""
    import cv2
    from pysift_b200.stitch import GPUPyStitch
    img1, img2, _ = synthetic.stitch_pair(600, 800, seed=8)
    kw = dict(ransac_iters=512, inlier_thresh=4.0, verbose=False)
    st = GPUPyStitch(max_dimension=640, denoise=True, sharpen=True, save_output=False, **kw)
    pano = st.stitch(img1, img2)

    def prep(im):
        im = cv2.resize(im, (640, 480), interpolation=cv2.INTER_AREA)
        im = cv2.bilateralFilter(im, d=9, sigmaColor=75, sigmaSpace=75)
        blur = cv2.GaussianBlur(im, (0, 0), sigmaX=2.0)
        return cv2.addWeighted(im, 1.5, blur, -0.5, 0)

    ref = GPUPyStitch(save_output=False, **kw).stitch(prep(img1), prep(img2))
    assert np.array_equal(pano, ref)
    monkeypatch.chdir(tmp_path)
    st2 = GPUPyStitch(output_max_dim=300, post_sharpen=True, save_output=True, **kw)
    out = st2.stitch(img1, img2)
    files = list(tmp_path.glob("panorama_*.png"))
    assert len(files) == 1
    saved = cv2.imread(str(files[0]))
    exp = out
    h, w = exp.shape[:2]
    if 300 / max(h, w) < 1.0:
        exp = cv2.resize(exp, (int(w * 300 / max(h, w)), int(h * 300 / max(h, w))), interpolation=cv2.INTER_AREA)
    exp = cv2.addWeighted(exp, 1.5, cv2.GaussianBlur(exp, (0, 0), sigmaX=2.0), -0.5, 0)
    assert np.array_equal(saved, exp)


@pytest.mark.parametrize("D,P", [(64, 32), (128, 128)])
def test_pca_basis_other_shapes_bit_exact(D, P):
    """The device Jacobi at the other compile-time dimension and all columns."""
    import torch
    from oracle import stitch_oracle as so
    L, lib = _lib()
    rng = np.random.default_rng(D + P)
    x = np.abs(rng.standard_normal((2000, D))).astype(np.float32) ** 2
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    _, cov = so.pca_stats(x)
    want, sweeps = so.pca_basis(cov, P, return_sweeps=True)
    c = torch.from_numpy(cov).cuda()
    sz = ctypes.c_size_t()
    assert lib.pysift_pca_basis_workspace_size(D, ctypes.byref(sz)) == 0
    ws = torch.empty(sz.value, dtype=torch.uint8, device="cuda")
    got = torch.empty((D, P), dtype=torch.float32, device="cuda")
    sw = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.pysift_pca_basis(c.data_ptr(), D, P, ws.data_ptr(), ws.numel(), got.data_ptr(), sw.data_ptr(),
                                _st()) == 0
    assert np.array_equal(got.cpu().numpy(), want)
    assert int(sw.item()) == sweeps


def test_ransac_with_device_count_equals_host_count():
    """pysift_ransac_count (the count read on the device, a larger capacity)
    gives pysift_ransac's H, mask and info bit for bit; a count below 4 gives
    the empty result without sampling."""
    import torch
    from oracle import stitch_oracle as so
    L, lib = _lib()
    p1, p2, _ = _correspondences(3)
    n, n_hyp, cap = len(p1), 1024, len(p1) + 37
    rnd = torch.from_numpy(so.mt19937_u32(42, 4 * n_hyp)).cuda()
    pad = lambda p: torch.from_numpy(np.vstack([p, np.full((cap - n, 2), 1e30)])).cuda()  # rows past n ignored
    d1, d2 = pad(p1), pad(p2)
    sz = ctypes.c_size_t()
    lib.pysift_ransac_workspace_size(cap, n_hyp, ctypes.byref(sz))
    ws = torch.empty(sz.value + 256, dtype=torch.uint8, device="cuda")
    off = (-ws.data_ptr()) % 256
    outs = []
    for dev_count in (False, True):
        H = torch.empty(9, dtype=torch.float64, device="cuda")
        mask = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        info = torch.empty(3, dtype=torch.int32, device="cuda")
        if dev_count:
            cnt = torch.tensor([n], dtype=torch.int32, device="cuda")
            rc = lib.pysift_ransac_count(d1.data_ptr(), d2.data_ptr(), cnt.data_ptr(), cap, rnd.data_ptr(), n_hyp,
                                         4.0, 4.0, 1, 10, ws.data_ptr() + off, sz.value, H.data_ptr(),
                                         mask.data_ptr(), info.data_ptr(), _st())
        else:
            rc = lib.pysift_ransac(d1.data_ptr(), d2.data_ptr(), n, rnd.data_ptr(), n_hyp, 4.0, 4.0, 1, 10,
                                   ws.data_ptr() + off, sz.value, H.data_ptr(), mask.data_ptr(), info.data_ptr(),
                                   _st())
        assert rc == 0
        outs.append((H.cpu().numpy(), mask[:n].cpu().numpy(), info.cpu().numpy()))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    assert outs[1][2][0] > 0.6 * n
    # three points on the device: the empty result
    cnt = torch.tensor([3], dtype=torch.int32, device="cuda")
    H = torch.ones(9, dtype=torch.float64, device="cuda")
    info = torch.full((3,), 7, dtype=torch.int32, device="cuda")
    mask = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    assert lib.pysift_ransac_count(d1.data_ptr(), d2.data_ptr(), cnt.data_ptr(), cap, rnd.data_ptr(), n_hyp, 4.0,
                                   4.0, 1, 10, ws.data_ptr() + off, sz.value, H.data_ptr(), mask.data_ptr(),
                                   info.data_ptr(), _st()) == 0
    assert np.array_equal(info.cpu().numpy(), [0, 0, 0]) and not H.cpu().numpy().any()


def test_stitch_replay_equals_eager():
    """The first call for the keypoint counts runs eagerly and captures the
    matcher + RANSAC launches, the next two replay them: all three give the
    same panorama, homography and inlier mask, and the replay equals the
    oracle."""
    from oracle import stitch_oracle as so
    from pysift_b200.stitch import GPUPyStitch
    img1, img2, _ = synthetic.stitch_pair(480, 640, seed=4)
    st = GPUPyStitch(ransac_iters=2048, inlier_thresh=4.0, save_output=False, verbose=False)
    runs = []
    for _ in range(3):
        pano = st.stitch(img1, img2)
        runs.append((pano.copy(), st._last["H"].copy(), st._last["mask"].cpu().numpy().copy()))
    assert len(st._graphs) == 1
    for pano, H, mask in runs[1:]:
        assert np.array_equal(pano, runs[0][0]) and np.array_equal(H, runs[0][1]) and np.array_equal(mask, runs[0][2])
    orc = so.OracleStitch(ransac_iters=2048, inlier_thresh=4.0).stitch(img1, img2)
    _assert_stitch_equals_oracle(st, runs[2][0], orc)


def test_stitch_replays_across_sizes_keep_their_buffers():
    """Pairs of two sizes, interleaved: each size's first call captures its
    own graph and later calls replay it after the other size ran (and
    allocated its own buffers) in between; every replay gives the result of
    that size's eager call."""
    from pysift_b200.stitch import GPUPyStitch
    pairs = [synthetic.stitch_pair(480, 640, seed=4)[:2], synthetic.stitch_pair(600, 800, seed=9)[:2]]
    st = GPUPyStitch(ransac_iters=2048, inlier_thresh=4.0, save_output=False, verbose=False)
    first = {}
    for rep in range(3):
        for i, (a, b) in enumerate(pairs):
            pano = st.stitch(a, b)
            got = (pano.copy(), st._last["H"].copy(), st._last["mask"].cpu().numpy().copy())
            if rep == 0:
                first[i] = got
            else:
                assert all(np.array_equal(x, y) for x, y in zip(got, first[i])), (rep, i)
    assert len(st._graphs) == 2
