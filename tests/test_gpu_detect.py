"""GPU parity of detectAndCompute against the CPU oracle (bit-exact).

The CUDA path runs through the C ABI (pysift_detect_and_compute) via the
PySIFT drop-in class; the oracle restates the reference's algorithm on the
CPU.  Every output row -- x, y, size, angle, response, octave and all 128
descriptor values -- must be identical, as must the Gaussian pyramid.
"""
import ctypes

import numpy as np
import pytest

from pysift_b200 import synthetic

pytestmark = pytest.mark.gpu


def _run_both(img, oracle_lib, **kw):
    import torch
    from pysift_b200 import PySIFT
    sift = PySIFT(**kw)
    out = sift.detect_arrays(img)
    okw = dict(kw)
    hv = okw.pop("high_vram", True)
    orc = oracle_lib.OracleSIFT(high_vram=hv, **okw)
    ref = orc.detect_and_compute(img)
    return sift, out, ref


def _pyramid_equal(sift, img, ref):
    import torch
    from pysift_b200 import _lib
    H, W = img.shape
    b = sift._bufs[(H, W)]
    lib = sift._lib
    ws = b.ws
    bad = []
    for o, g in enumerate(ref["pyramid"]):
        for s in range(g.shape[0]):
            off, rows, cols, pitch = ctypes.c_size_t(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
            rc = lib.pysift_detect_workspace_view(ctypes.byref(sift._cfg), H, W, 0, o, s, ctypes.byref(off),
                                                  ctypes.byref(rows), ctypes.byref(cols), ctypes.byref(pitch))
            assert rc == 0
            start = b.ws_off + off.value
            n = rows.value * pitch.value * 4
            arr = ws[start:start + n].view(torch.float32).view(rows.value, pitch.value)[:, :cols.value].cpu().numpy()
            if not np.array_equal(arr, g[s]):
                d = np.abs(arr - g[s])
                bad.append((o, s, float(d.max()), int((d > 0).sum())))
    return bad


def _compare(out, ref):
    n_gpu, n_ref = len(out["x"]), len(ref["x"])
    assert n_gpu == n_ref, f"keypoint count {n_gpu} != oracle {n_ref}"
    for k in ("x", "y", "size", "angle", "response", "octave"):
        a, b = out[k], ref[k]
        assert np.array_equal(a, b), f"{k}: {int(np.sum(a != b))} rows differ"
    d = out["desc"]
    assert np.array_equal(d, ref["desc"]), f"desc: max diff {np.abs(d - ref['desc']).max()}"


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_cfg1_scene_bit_exact(seed, oracle_lib):
    img = synthetic.scene(480, 640, seed=seed)
    sift, out, ref = _run_both(img, oracle_lib)
    bad = _pyramid_equal(sift, img, ref)
    assert not bad, f"pyramid levels differ (octave, level, max|d|, count): {bad[:6]}"
    st = sift.last_stats
    assert st[1] == ref["n_refined"] or ref["capped"]
    _compare(out, ref)


@pytest.mark.parametrize("shape", [(37, 53), (12, 16), (121, 90)])
def test_odd_sizes(shape, oracle_lib):
    img = synthetic.scene(shape[0], shape[1], seed=7)
    sift, out, ref = _run_both(img, oracle_lib)
    assert not _pyramid_equal(sift, img, ref)
    _compare(out, ref)


def test_wide_image_bit_exact(oracle_lib):
    """1024 x 2100: doubled (8.6 Mpix, under the cap), so the in-place row
    prefilter walks each 2100-wide row in two chunks, and the blur tile
    heights are picked for odd level sizes; pyramid and every output row
    bit-exact against the oracle."""
    img = synthetic.scene(1024, 2100, seed=9)
    sift, out, ref = _run_both(img, oracle_lib)
    assert sift.last_stats[5] == 1
    assert not _pyramid_equal(sift, img, ref)
    _compare(out, ref)


def test_no_doubling(oracle_lib):
    img = synthetic.scene(480, 640, seed=3)
    sift, out, ref = _run_both(img, oracle_lib, double_image=False)
    assert sift.last_stats[5] == 0
    _compare(out, ref)


def test_fp16_dsp_low_vram_tier(oracle_lib):
    """The configuration of the reference's golden dumps: 4 octaves, fp16
    pyramid, DSP-5 descriptors, 4 MP doubling cap."""
    img = synthetic.scene(300, 400, seed=4)
    sift, out, ref = _run_both(img, oracle_lib, n_octaves=4, dsp=True, dsp_n_scales=5, fp16_pyramid=True,
                               high_vram=False)
    assert not _pyramid_equal(sift, img, ref)
    _compare(out, ref)


def test_starvation_retry(oracle_lib):
    """Few keypoints -> the half-threshold retry runs (pysift/core.py:2066-2071)."""
    H, W = 200, 240
    yy, xx = np.mgrid[0:H, 0:W]
    img = (128 + 60 * np.exp(-((yy - 100) ** 2 + (xx - 120) ** 2) / (2 * 20.0 ** 2))).astype(np.uint8)
    sift, out, ref = _run_both(img, oracle_lib)
    assert ref["retried"]
    assert sift.last_stats[3] == 1
    _compare(out, ref)


def test_candidate_cap_overflow(oracle_lib):
    """An octave with more than 25,000 extrema (pysift/core.py:1395, 209-214):
    the first 25,000 in (scale, row, column) order are refined, the overflow
    is reported in the stats, and every output row equals the oracle's."""
    img = synthetic.dense_texture(900, 1200, seed=6, sigma=1.0)
    sift, out, ref = _run_both(img, oracle_lib)
    assert ref["n_cands"][0] > 25000
    st = sift.last_stats
    assert st[6] >= 1
    assert list(st[8:8 + len(ref["n_cands"])]) == list(ref["n_cands"])
    _compare(out, ref)


def test_keypoint_cap(oracle_lib):
    """More than 8000 refined keypoints -> top-8000 by response (pysift/core.py:2078-2080)."""
    img = synthetic.dense_texture(800, 1000, seed=5, sigma=2.0)
    sift, out, ref = _run_both(img, oracle_lib)
    assert ref["capped"]
    assert sift.last_stats[4] == 1
    _compare(out, ref)


def test_device_input_and_gpu_output(oracle_lib):
    import torch
    from pysift_b200 import PySIFT
    img = synthetic.scene(240, 320, seed=9)
    sift = PySIFT()
    kp_t, desc_t = sift.detectAndCompute(torch.from_numpy(img).cuda(), gpu_output=True)
    assert kp_t.is_cuda and desc_t.is_cuda and kp_t.shape[1] == 4 and desc_t.shape[1] == 128
    ref = oracle_lib.OracleSIFT().detect_and_compute(img)
    assert kp_t.shape[0] == len(ref["x"])
    assert np.array_equal(kp_t[:, 0].cpu().numpy(), ref["x"])
    assert np.array_equal(desc_t.cpu().numpy(), ref["desc"])
    kps, desc = sift.detectAndCompute(img)
    assert len(kps) == len(ref["x"]) and desc.shape == (len(ref["x"]), 128)
    assert kps[0].pt == (float(ref["x"][0]), float(ref["y"][0]))


def test_repeat_determinism():
    from pysift_b200 import PySIFT
    img = synthetic.scene(480, 640, seed=11)
    sift = PySIFT()
    a = sift.detect_arrays(img)
    b = sift.detect_arrays(img)
    for k in a:
        assert np.array_equal(a[k], b[k])


@pytest.mark.parametrize("limit", [500, 100000])
def test_output_limit_is_stable_topk_by_response(limit):
    """output_limit = N keeps the N largest responses, ordered by response
    with ties in (x, y) order, exactly as a stable top-N of the full output."""
    import torch
    from pysift_b200 import PySIFT
    img = synthetic.dense_texture(480, 640, seed=5, sigma=2.0)
    full = PySIFT()
    kp, desc = full.detectAndCompute(img, gpu_output=True)
    n = kp.shape[0]
    resp = full._buffers(480, 640).resp[:n].cpu().numpy()
    lim = PySIFT()
    lim._cfg.output_limit = limit
    kp2, desc2 = lim.detectAndCompute(img, gpu_output=True)
    if n > limit:
        order = np.argsort(-resp, kind="stable")[:limit]
    else:
        order = np.arange(n)
    assert kp2.shape[0] == len(order)
    assert np.array_equal(kp2.cpu().numpy(), kp.cpu().numpy()[order])
    assert np.array_equal(desc2.cpu().numpy(), desc.cpu().numpy()[order])
    assert np.array_equal(lim._buffers(480, 640).resp[:len(order)].cpu().numpy(), resp[order])


@pytest.mark.parametrize("sigma", [0.0, 1.2, 3.0, 4.0, 5.0])
@pytest.mark.parametrize("H,W,pitch", [(257, 301, 301), (200, 320, 331), (130, 128, 160)])
def test_gauss_blur_entry_point(sigma, H, W, pitch, oracle_lib):
    """pysift_gauss_blur with caller pitches (odd and even) against the
    oracle's sequential FMA-chain blur, bit for bit; radii 0 (copy), 5, 12,
    16 and 20 (the general kernel)."""
    import torch
    from oracle import oracle
    from pysift_b200 import _lib
    from pysift_b200.core import gaussian_weights
    lib = _lib.load()
    rng = np.random.default_rng(H * W + int(sigma * 10))
    img = rng.random((H, W), dtype=np.float32)
    src = torch.zeros((H, pitch), dtype=torch.float32, device="cuda")
    src[:, :W] = torch.from_numpy(img).cuda()
    dst = torch.full((H, pitch), float("nan"), dtype=torch.float32, device="cuda")
    k, radius = gaussian_weights(sigma) if sigma > 0 else (np.ones(1, np.float32), 0)
    k = np.ascontiguousarray(k, dtype=np.float32)
    rc = lib.pysift_gauss_blur(src.data_ptr(), pitch, dst.data_ptr(), pitch, H, W,
                               k.ctypes.data_as(ctypes.c_void_p), radius, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.pysift_last_error()
    ref = oracle.gauss_blur(img, sigma) if sigma > 0 else img
    assert np.array_equal(dst[:, :W].cpu().numpy(), ref)


@pytest.mark.parametrize("rows", [16, 32, 40])
def test_gauss_blur_every_tile_height(rows, oracle_lib):
    """Each register-blocked blur variant (tile height forced through the
    testing hook; normally picked per launch from the level size and the
    occupancy) against the oracle's FMA-chain blur, bit for bit, for radii
    1, 5, 12 and 16 and odd and even pitches."""
    import torch
    from oracle import oracle
    from pysift_b200 import _lib
    from pysift_b200.core import gaussian_weights
    lib = _lib.load()
    assert lib.pysift_set_blur_tile_rows(7) != 0  # only 0, 16, 32 and 40
    try:
        assert lib.pysift_set_blur_tile_rows(rows) == 0
        for sigma, (H, W, pitch) in [(0.3, (75, 130, 131)), (1.25, (257, 301, 301)), (3.0, (130, 128, 160)),
                                     (4.0, (90, 200, 203))]:
            rng = np.random.default_rng(H * W + rows)
            img = rng.random((H, W), dtype=np.float32)
            src = torch.zeros((H, pitch), dtype=torch.float32, device="cuda")
            src[:, :W] = torch.from_numpy(img).cuda()
            dst = torch.full((H, pitch), float("nan"), dtype=torch.float32, device="cuda")
            k, radius = gaussian_weights(sigma)
            k = np.ascontiguousarray(k, dtype=np.float32)
            rc = lib.pysift_gauss_blur(src.data_ptr(), pitch, dst.data_ptr(), pitch, H, W,
                                       k.ctypes.data_as(ctypes.c_void_p), radius,
                                       torch.cuda.current_stream().cuda_stream)
            assert rc == 0, lib.pysift_last_error()
            assert np.array_equal(dst[:, :W].cpu().numpy(), oracle.gauss_blur(img, sigma)), (sigma, radius)
    finally:
        lib.pysift_set_blur_tile_rows(0)


def test_detect_batch_matches_single_image_calls():
    """detect_batch on uneven sizes over several streams returns, per image,
    exactly what detectAndCompute returns for that image alone."""
    from pysift_b200 import PySIFT
    sizes = [(240, 320), (361, 479), (480, 640), (200, 300), (333, 517), (480, 640), (97, 131)]
    imgs = [synthetic.scene(h, w, seed=30 + i) for i, (h, w) in enumerate(sizes)]
    sift = PySIFT()
    ref = [sift.detectAndCompute(im, gpu_output=True) for im in imgs]
    for n_streams in (3, 1):
        got = sift.detect_batch(imgs, n_streams=n_streams)
        assert len(got) == len(imgs)
        for (k1, d1), (k2, d2) in zip(ref, got):
            assert np.array_equal(k1.cpu().numpy(), k2.cpu().numpy())
            assert np.array_equal(d1.cpu().numpy(), d2.cpu().numpy())
    host = sift.detect_batch(imgs[:3], n_streams=2, gpu_output=False)
    assert np.array_equal(host[1][1], ref[1][1].cpu().numpy())


def test_as_uint8_descriptors_and_exact_matching(oracle_lib):
    """PySIFT(rootsift=False, as_uint8=True): OpenCV's uint8 form
    saturate(rint(512 v)) of the oracle's L2 / clip / L2 descriptors, bit for
    bit, through detectAndCompute and detect_batch; the uint8 sets of two
    views then match exactly (BF16 tcgen05 path) like the int64 oracle."""
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import PySIFT, match
    img1, img2, _ = synthetic.stitch_pair(480, 640, seed=4)
    import cv2
    g1 = cv2.cvtColor(img1, cv2.COLOR_BGR2GRAY)
    g2 = cv2.cvtColor(img2, cv2.COLOR_BGR2GRAY)
    sift = PySIFT(rootsift=False, as_uint8=True)
    orc = oracle_lib.OracleSIFT(rootsift=False)
    outs = []
    for g in (g1, g2):
        kps, desc = sift.detectAndCompute(g)
        ref = orc.detect_and_compute(g)
        ref_u8 = np.clip(np.rint(ref["desc"] * np.float32(512.0)), 0, 255).astype(np.uint8)
        assert desc.dtype == np.uint8 and np.array_equal(desc, ref_u8)
        assert len(kps) == len(ref["x"])
        outs.append(desc)
    batch = sift.detect_batch([g1, g2], gpu_output=False)
    for (k, d), ref in zip(batch, outs):
        assert np.array_equal(d, ref)
    a = torch.from_numpy(outs[0]).cuda()
    b = torch.from_numpy(outs[1]).cuda()
    m = match.match_u8_exact(a, b, 0.75)
    n = int(m["count"].item())
    ref = mo.match_u8_exact(outs[0], outs[1], 0.75)
    assert n == len(ref["pairs"]) and n > 20
    assert np.array_equal(m["pairs"][:n].cpu().numpy(), ref["pairs"])
    dm = match.to_dmatches(m)
    assert len(dm) == n and dm[0].queryIdx == int(ref["pairs"][0, 0]) and dm[0].trainIdx == int(ref["pairs"][0, 1])


def test_detect_batch_graph_replay_matches_eager():
    """detect_batch(graph=True): the batch captured once as a CUDA graph and
    replayed on new images of the same sizes gives exactly the eager results."""
    from pysift_b200 import PySIFT
    sizes = [(480, 640), (360, 480), (600, 800), (480, 640), (300, 400)]
    sift = PySIFT()
    first = [synthetic.scene(h, w, seed=30 + i) for i, (h, w) in enumerate(sizes)]
    second = [synthetic.scene(h, w, seed=60 + i) for i, (h, w) in enumerate(sizes)]
    for imgs in (first, second, first):
        eager = sift.detect_batch(imgs, n_streams=4, gpu_output=False)
        graph = sift.detect_batch(imgs, n_streams=4, gpu_output=False, graph=True)
        assert len(eager) == len(graph)
        for (k1, d1), (k2, d2) in zip(eager, graph):
            assert k1.shape[0] > 0 and np.array_equal(k1, k2) and np.array_equal(d1, d2)


def test_single_image_graph_replay(oracle_lib):
    """detectAndCompute replays a captured CUDA graph from the second call on
    (per size): results equal the eager instance's and the oracle's, and each
    replay adds the same number of launches to the library's count as an
    eager call."""
    from pysift_b200 import PySIFT, _lib
    lib = _lib.load()
    a = synthetic.scene(480, 640, seed=41)
    b = synthetic.scene(480, 640, seed=42)
    eager = PySIFT(graphs=False)
    graph = PySIFT()
    for img in (a, b, a, b):
        n0 = lib.pysift_launch_count()
        k1, d1 = eager.detectAndCompute(img, gpu_output=True)
        n1 = lib.pysift_launch_count()
        k2, d2 = graph.detectAndCompute(img, gpu_output=True)
        n2 = lib.pysift_launch_count()
        assert torch_equal(k1, k2) and torch_equal(d1, d2)
        assert n2 - n1 == n1 - n0
    ref = oracle_lib.OracleSIFT().detect_and_compute(b)
    assert np.array_equal(d2.cpu().numpy(), ref["desc"])


def test_capture_on_a_stream_the_library_has_not_seen():
    """A detection captured into a CUDA graph on a fresh stream with no eager
    call on that stream first (the library then keeps all of its work on the
    caller's stream instead of forking its side stream): the replay's rows
    equal an eager detection's."""
    import torch
    from pysift_b200 import PySIFT, _lib
    img = synthetic.scene(480, 640, seed=43)
    k1, d1 = PySIFT(graphs=False).detectAndCompute(img, gpu_output=True)
    sift = PySIFT(graphs=False)
    H, W = img.shape
    g_dev = torch.from_numpy(img).cuda()
    b = sift._buffers(H, W)  # allocated outside the capture
    torch.cuda.synchronize()
    fresh = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=fresh):
        sift._launch(b, g_dev.data_ptr(), H, W, W, fresh.cuda_stream)
    graph.replay()
    torch.cuda.synchronize()
    n = int(b.stats.cpu()[_lib.STAT_N_KEYPOINTS])
    assert n == k1.shape[0] and n > 0
    assert torch_equal(b.kpts[:n], k1) and torch_equal(b.desc[:n], d1)


def torch_equal(x, y):
    import torch
    return x.shape == y.shape and bool(torch.equal(x, y))
