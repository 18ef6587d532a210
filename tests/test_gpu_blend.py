"""GPU parity of the reference composition (gain, DP seam, multiband blend,
paste): bit-exact against the reference's own output on the golden canvases
and against the oracle (oracle/blend_oracle.py) on larger seeded canvases,
and inside GPUPyStitch."""
import os

import numpy as np
import pytest

from pysift_b200 import synthetic

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "blend_cases.npz")


def _run(w1, m1, c2, m2, n_levels=6, color_match="gain"):
    import torch
    from pysift_b200 import blend
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    pano, both, rmse, _ = blend.blend_multiband(t(w1), t(m1.astype(np.uint8)), t(c2), t(m2.astype(np.uint8)), n_levels,
                                                color_match=color_match)
    torch.cuda.synchronize()
    return pano.cpu().numpy(), both.cpu().numpy().astype(bool), float(rmse.cpu()[0])


def _rmse(w1, m1, c2, m2):
    """_seam_rmse of the gained image 1 (pysift/core.py:3555-3562), exact."""
    from oracle import blend_oracle as bo
    ov = m1 & m2
    if not ov.any():
        return float("nan")
    g = bo.gain_compensate(w1.astype(np.float32), c2.astype(np.float32), ov)
    d = g.astype(np.uint8)[ov].astype(np.int64) - c2[ov].astype(np.int64)
    return float(np.sqrt((d * d).sum() / d.size))


def _case(seed, ch, cw, stacked=False, flip=False):
    """Seeded canvas: a projective quad for image 1, a rectangle for image 2,
    textured images with a colour gain between them and stray values of the
    warp outside image 1's mask."""
    rng = np.random.default_rng(seed)
    # masks are drawn side by side; a stacked canvas draws them transposed
    yy, xx = np.mgrid[0:cw, 0:ch] if stacked else np.mgrid[0:ch, 0:cw]
    yy, xx = yy.astype(np.float64), xx.astype(np.float64)
    L = xx.shape[1]
    k = rng.uniform(-0.15, 0.15)
    m1 = (xx < 0.62 * L + k * (yy - yy.mean())) & (yy > 0.03 * yy.max() + 0.02 * xx)
    m2 = (xx >= 0.38 * L) & (yy >= 2) & (yy < yy.max() - 1)
    if stacked:
        m1, m2 = m1.T.copy(), m2.T.copy()
    if flip:
        m1, m2 = m1[:, ::-1].copy(), m2[:, ::-1].copy()
    base = synthetic.dense_texture(ch, cw, seed=seed).astype(np.float64)
    g1 = rng.uniform(0.6, 1.3, 3)
    w1 = np.clip(base[:, :, None] * g1 + rng.normal(0, 3, (ch, cw, 3)), 0, 255).astype(np.uint8)
    c2 = np.clip(base[:, :, None] * rng.uniform(0.8, 1.2, 3) + rng.normal(0, 3, (ch, cw, 3)), 0, 255).astype(np.uint8)
    stray = (~m1) & (rng.random((ch, cw)) < 0.03)
    w1[~m1] = 0
    w1[stray] = 41
    c2[~m2] = 0
    return w1, m1, c2, m2


def test_blend_reference_golden_bit_exact():
    g = np.load(GOLDEN)
    for name in g["names"]:
        w1, m1, c2, m2 = (g[f"{name}_{k}"] for k in ("warped1", "mask1", "canvas2", "mask2"))
        pano, both, rmse = _run(w1, m1, c2, m2)
        assert np.array_equal(both, g[f"{name}_both"]), name
        assert np.array_equal(pano, g[f"{name}_pano"]), name
        ref = float(g[f"{name}_seam_rmse"])
        if np.isnan(ref):
            assert np.isnan(rmse)
        else:
            assert abs(rmse - ref) <= 1e-5 * ref, (name, rmse, ref)


@pytest.mark.parametrize("seed,ch,cw,stacked,flip", [
    (1, 300, 520, False, False),
    (2, 300, 520, False, True),
    (3, 520, 300, True, False),
    (4, 257, 611, False, False),
    (5, 611, 257, True, True),
    (6, 720, 1300, False, False),
    (8, 900, 2100, False, True),
])
def test_blend_matches_oracle(seed, ch, cw, stacked, flip):
    from oracle import blend_oracle as bo
    w1, m1, c2, m2 = _case(seed, ch, cw, stacked, flip)
    pano, both, rmse = _run(w1, m1, c2, m2)
    ref, ref_both = bo.blend_pair(w1, m1, c2, m2)
    assert np.array_equal(both, ref_both)
    assert np.array_equal(pano, ref), np.argwhere(pano != ref)[:5]
    assert abs(rmse - _rmse(w1, m1, c2, m2)) <= 1e-12 * max(1.0, rmse)


@pytest.mark.parametrize("n_levels", [1, 2, 3, 5])
def test_blend_levels(n_levels):
    from oracle import blend_oracle as bo
    w1, m1, c2, m2 = _case(11, 190, 333)
    pano, _, _ = _run(w1, m1, c2, m2, n_levels)
    ref, _ = bo.blend_pair(w1, m1, c2, m2, n_levels=n_levels)
    assert np.array_equal(pano, ref)


@pytest.mark.parametrize("cw", [4000, 5000, 9000, 13000])
def test_blend_long_canvas(cw):
    """A vertical seam across wide canvases: the DP lines in shared memory with
    a 4-deep cost ring or without one, and in global memory."""
    from oracle import blend_oracle as bo
    ch = 90
    rng = np.random.default_rng(cw)
    yy, xx = np.mgrid[0:ch, 0:cw]
    a = cw // 2
    m1 = xx < a + 20 + yy // 8
    m2 = (xx >= a - 25) & (yy >= 3)
    base = synthetic.dense_texture(ch, cw, seed=cw).astype(np.float64)
    w1 = np.clip(base[:, :, None] * 0.8 + rng.normal(0, 3, (ch, cw, 3)), 0, 255).astype(np.uint8)
    c2 = np.clip(base[:, :, None] * 1.1 + rng.normal(0, 3, (ch, cw, 3)), 0, 255).astype(np.uint8)
    w1[~m1] = 0
    c2[~m2] = 0
    pano, both, _ = _run(w1, m1, c2, m2)
    ref, ref_both = bo.blend_pair(w1, m1, c2, m2)
    assert np.array_equal(both, ref_both)
    assert np.array_equal(pano, ref)


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_blend_degenerate_masks(seed):
    """Overlaps with holes, disconnected parts and lines far apart: the DP
    window logic and the backtrack through INF positions."""
    from oracle import blend_oracle as bo
    rng = np.random.default_rng(100 + seed)
    ch, cw = 120, 170
    m1 = rng.random((ch, cw)) < (0.3 + 0.1 * seed)
    m2 = rng.random((ch, cw)) < 0.5
    if seed % 2:
        m1[:, : cw // 3] = True
        m2[: ch // 2, cw // 2:] = True
    w1 = rng.integers(0, 256, (ch, cw, 3), dtype=np.uint8)
    c2 = rng.integers(0, 256, (ch, cw, 3), dtype=np.uint8)
    w1[~m1] = 0
    c2[~m2] = 0
    pano, both, _ = _run(w1, m1, c2, m2)
    ref, ref_both = bo.blend_pair(w1, m1, c2, m2)
    assert np.array_equal(both, ref_both)
    assert np.array_equal(pano, ref)


def test_blend_no_overlap_and_edges():
    """No overlap (no gain, no seam), an overlap of one column and one of one row."""
    from oracle import blend_oracle as bo
    ch, cw = 64, 97
    rng = np.random.default_rng(3)
    w1 = rng.integers(0, 256, (ch, cw, 3), dtype=np.uint8)
    c2 = rng.integers(0, 256, (ch, cw, 3), dtype=np.uint8)
    yy, xx = np.mgrid[0:ch, 0:cw]
    for m1, m2 in [(xx < 40, xx >= 50), (xx <= 48, xx >= 48), (yy <= 30, yy >= 30), (xx >= 0, xx >= 0)]:
        a, b = w1.copy(), c2.copy()
        a[~m1] = 0
        b[~m2] = 0
        pano, both, _ = _run(a, m1, b, m2)
        ref, ref_both = bo.blend_pair(a, m1, b, m2)
        assert np.array_equal(pano, ref) and np.array_equal(both, ref_both)


def test_stitch_multiband_compose_bit_exact():
    """GPUPyStitch's default composition equals the oracle on the warp the
    stitcher made, and image 2's canvas is the reference's paste."""
    from oracle import blend_oracle as bo
    from pysift_b200.stitch import GPUPyStitch
    img1, img2, _ = synthetic.stitch_pair(480, 640, seed=1)
    st = GPUPyStitch(ransac_iters=2048, inlier_thresh=4.0, save_output=False, verbose=False)
    pano = st.stitch(img1, img2)
    c = st._last_compose
    ch, cw = c["canvas_h"], c["canvas_w"]
    w1 = c["warped1"].cpu().numpy()
    m1 = c["mask1"].cpu().numpy().astype(bool)
    m2 = c["mask2"].cpu().numpy().astype(bool)
    c2 = c["canvas2"].cpu().numpy()
    iox, ioy = int(round(c["ox"])), int(round(c["oy"]))
    ref_c2 = np.zeros((ch, cw, 3), np.uint8)
    ye, xe = min(ioy + img2.shape[0], ch), min(iox + img2.shape[1], cw)
    ref_c2[ioy:ye, iox:xe] = img2[:ye - ioy, :xe - iox]
    assert np.array_equal(c2, ref_c2)
    ref, _ = bo.blend_pair(w1, m1, c2, m2)
    assert np.array_equal(c["out"].cpu().numpy(), ref)
    assert pano.ndim == 3 and pano.shape[2] == 3
    assert np.isfinite(st.last_metrics["seam_rmse"])
    assert abs(st.last_metrics["seam_rmse"] - _rmse(w1, m1, c2, m2)) < 1e-9


def test_stitch_multiband_end_to_end():
    from oracle import stitch_oracle as so
    from pysift_b200.stitch import GPUPyStitch
    img1, img2, _ = synthetic.stitch_pair(480, 640, seed=2)
    st = GPUPyStitch(ransac_iters=2048, inlier_thresh=4.0, save_output=False, verbose=False)
    pano = st.stitch(img1, img2)
    orc = so.OracleStitch(ransac_iters=2048, inlier_thresh=4.0).stitch(img1, img2)
    assert np.array_equal(st._last["pairs"].cpu().numpy(), orc["pairs"])
    assert np.array_equal(st._last["mask"].cpu().numpy().astype(bool), orc["mask"])
    assert np.array_equal(st._last["H"], orc["H"])
    c = st._last_compose
    assert (c["canvas_w"], c["canvas_h"]) == orc["canvas_size"]
    assert np.array_equal(c["out"].cpu().numpy(), orc["canvas"])
    assert pano.shape == orc["pano"].shape and np.array_equal(pano, orc["pano"])


TRIPLES = os.path.join(os.path.dirname(__file__), "golden", "triple_cases.npz")


def test_float_image_blend_and_triple_composition():
    """The two-pass composition of _stitch_triple on the reference's own
    canvases: pass 1's unclipped float blend equals the oracle's float32
    output bit for bit, pass 2 (float image 1) gives the oracle's panorama,
    and after the crop the reference's own panorama within one level on a
    few values (the second pass's float gain mean)."""
    import torch
    from oracle import blend_oracle as bo
    from oracle import stitch_oracle as so
    from pysift_b200 import blend
    g = np.load(TRIPLES)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    for name in g["names"]:
        w1, m1, c2, m2, w3, m3 = (g[f"{name}_{k}"] for k in ("warped1", "mask1", "canvas2", "mask2", "warped3",
                                                             "mask3"))
        ch, cw = m1.shape
        b12 = torch.empty((ch, cw, 3), dtype=torch.float32, device="cuda")
        _, m12, r12, _ = blend.blend_multiband(t(w1), t(m1.astype(np.uint8)), t(c2), t(m2.astype(np.uint8)),
                                               blended=b12, want_pano=False)
        ref_b12, ref_m12, ref_r12 = bo.blend_core(w1.astype(np.float32), m1, c2.astype(np.float32), m2)
        assert np.array_equal(b12.cpu().numpy(), ref_b12)
        assert np.array_equal(m12.cpu().numpy().astype(bool), ref_m12)
        pano, both, r23, _ = blend.blend_multiband(b12, m12, t(w3), t(m3.astype(np.uint8)))
        torch.cuda.synchronize()
        ref_pano, ref_both, _, ref_r23 = bo.compose3(w1, m1, c2, m2, w3, m3)
        assert np.array_equal(pano.cpu().numpy(), ref_pano)
        assert np.array_equal(both.cpu().numpy().astype(bool), ref_both)
        assert abs(float(r12.cpu()[0]) - ref_r12) < 1e-12 and abs(float(r23.cpu()[0]) - ref_r23) < 1e-12
        ext = blend.mask_extents(both).cpu().numpy()
        bb = ref_both
        rows_lo = np.where(bb.any(1), bb.argmax(1), 0x7fffffff)
        rows_hi = np.where(bb.any(1), cw - 1 - bb[:, ::-1].argmax(1), -1)
        cols_lo = np.where(bb.any(0), bb.argmax(0), 0x7fffffff)
        cols_hi = np.where(bb.any(0), ch - 1 - bb[::-1, :].argmax(0), -1)
        assert np.array_equal(ext, np.concatenate([rows_lo, rows_hi, cols_lo, cols_hi]).astype(np.int32))
        crop = so.autocrop(pano.cpu().numpy(), ref_both)
        d = np.abs(crop.astype(int) - g[f"{name}_pano"].astype(int))
        assert d.max() <= 1 and (d > 0).mean() < 5e-4


@pytest.mark.parametrize("int8", [False, True])
def test_stitch_three_images_end_to_end(int8):
    """GPUPyStitch.stitch(img1, img2, img3) against the oracle's
    _stitch_triple restatement: the same matches, homographies and panorama."""
    from oracle import stitch_oracle as so
    from pysift_b200.stitch import GPUPyStitch
    a, b, c, H12, H32 = synthetic.stitch_triple(360, 480, seed=1)
    st = GPUPyStitch(ransac_iters=1024, inlier_thresh=4.0, save_output=False, verbose=False, int8_matching=int8)
    pano = st.stitch(a, b, c)
    orc = so.OracleStitch(ransac_iters=1024, inlier_thresh=4.0, int8_matching=int8).stitch3(a, b, c)
    m = st.last_metrics
    assert m["matches_12"] == len(orc["pairs12"]) and m["matches_23"] == len(orc["pairs23"])
    assert np.array_equal(st._last["pairs12"].cpu().numpy(), orc["pairs12"])
    assert np.array_equal(st._last["pairs23"].cpu().numpy(), orc["pairs23"])
    assert np.array_equal(st._last["H12"], orc["H12"]) and np.array_equal(st._last["H32"], orc["H32"])
    assert (m["canvas_w"], m["canvas_h"]) == orc["canvas"]
    assert pano.shape == orc["pano"].shape and np.array_equal(pano, orc["pano"])
    assert abs(m["seam_rmse"] - orc["rmse12"]) < 1e-9 and abs(m["seam_rmse_23"] - orc["rmse23"]) < 1e-9
    H12n = H12 / H12[2, 2]
    assert np.allclose(st._last["H12"] / st._last["H12"][2, 2], H12n, rtol=2e-2, atol=2e-2 * np.abs(H12n).max())
    Hc = np.linalg.inv(st._last["H32"]) @ st._last["H12"]
    Hc /= Hc[2, 2]
    assert abs(m["chain_scale"] - np.sqrt(abs(np.linalg.det(Hc[:2, :2])))) < 1e-12
    assert abs(m["chain_rotation_deg"] - np.degrees(np.arctan2(Hc[1, 0], Hc[0, 0]))) < 1e-9


def test_histogram_matching():
    """color_match='hist' (_hist_match, pysift/core.py:3591-3625): bit-exact
    against the oracle on the golden canvases and seeded canvases, with a
    float image 1 too (the second pass of a three-image stitch); against the
    reference's own output within one level (the canonical seam blur)."""
    import torch
    from oracle import blend_oracle as bo
    from pysift_b200 import blend
    g = np.load(GOLDEN)
    for name in g["names"]:
        w1, m1, c2, m2 = (g[f"{name}_{k}"] for k in ("warped1", "mask1", "canvas2", "mask2"))
        pano, both, rmse = _run(w1, m1, c2, m2, color_match="hist")
        ref, _ = bo.blend_pair(w1, m1, c2, m2, color_match="hist")
        assert np.array_equal(pano, ref), name
        d = np.abs(pano.astype(int) - g[f"{name}_hist_pano"].astype(int))
        assert d.max() <= 1 and (d > 0).mean() < 1e-3
    for args in [(21, 300, 520, False, False), (22, 520, 300, True, True)]:
        w1, m1, c2, m2 = _case(*args)
        pano, _, rmse = _run(w1, m1, c2, m2, color_match="hist")
        ref, _ = bo.blend_pair(w1, m1, c2, m2, color_match="hist")
        assert np.array_equal(pano, ref)
    g = np.load(TRIPLES)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    for name in g["names"]:
        w1, m1, c2, m2, w3, m3 = (g[f"{name}_{k}"] for k in ("warped1", "mask1", "canvas2", "mask2", "warped3",
                                                             "mask3"))
        ch, cw = m1.shape
        b12 = torch.empty((ch, cw, 3), dtype=torch.float32, device="cuda")
        _, m12, _, _ = blend.blend_multiband(t(w1), t(m1.astype(np.uint8)), t(c2), t(m2.astype(np.uint8)),
                                             blended=b12, want_pano=False, color_match="hist")
        pano, _, _, _ = blend.blend_multiband(b12, m12, t(w3), t(m3.astype(np.uint8)), color_match="hist")
        ref, _, _, _ = bo.compose3(w1, m1, c2, m2, w3, m3, color_match="hist")
        assert np.array_equal(pano.cpu().numpy(), ref), name


def test_stitch_color_match_hist_end_to_end():
    """GPUPyStitch(color_match='hist'): the composed canvas equals the
    oracle's composition of the stitcher's own warp."""
    from oracle import blend_oracle as bo
    from pysift_b200.stitch import GPUPyStitch
    img1, img2, _ = synthetic.stitch_pair(480, 640, seed=3)
    st = GPUPyStitch(ransac_iters=1024, inlier_thresh=4.0, save_output=False, verbose=False, color_match="hist")
    st.stitch(img1, img2)
    c = st._last_compose
    ref, _ = bo.blend_pair(c["warped1"].cpu().numpy(), c["mask1"].cpu().numpy().astype(bool),
                           c["canvas2"].cpu().numpy(), c["mask2"].cpu().numpy().astype(bool), color_match="hist")
    assert np.array_equal(c["out"].cpu().numpy(), ref)


@pytest.mark.parametrize("ch,cw,ov_lo,ov_hi", [(1100, 1500, 500, 1400), (1500, 1900, 300, 1750),
                                                (2150, 2500, 200, 2330)])
def test_blend_wide_overlap_bands(ch, cw, ov_lo, ov_hi):
    """Wide overlap bands (~900 and ~1470 columns for a vertical seam, ~2150
    rows for a horizontal one): windows of a thousand and more positions per
    DP line."""
    from oracle import blend_oracle as bo
    rng = np.random.default_rng(cw)
    yy, xx = np.mgrid[0:ch, 0:cw]
    m1 = xx < ov_hi + (yy * 0.04).astype(int) - 40
    m2 = (xx >= ov_lo + (yy * 0.03).astype(int)) & (yy >= 2)
    base = synthetic.dense_texture(ch, cw, seed=ch).astype(np.float64)
    w1 = np.clip(base[:, :, None] * 0.9 + rng.normal(0, 3, (ch, cw, 3)), 0, 255).astype(np.uint8)
    c2 = np.clip(base[:, :, None] * 1.05 + rng.normal(0, 3, (ch, cw, 3)), 0, 255).astype(np.uint8)
    w1[~m1] = 0
    c2[~m2] = 0
    pano, both, _ = _run(w1, m1, c2, m2)
    ref, ref_both = bo.blend_pair(w1, m1, c2, m2)
    assert np.array_equal(both, ref_both)
    assert np.array_equal(pano, ref)


def test_blend_in_a_cuda_graph():
    """The composition captures into a CUDA graph (no host copies or syncs
    inside, the side stream forked and joined): replays on new canvases of the
    same size give the eager results."""
    import torch
    from pysift_b200 import blend
    w1, m1, c2, m2 = _case(31, 240, 400)
    w1b, _, c2b, _ = _case(32, 240, 400)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    W1, M1, C2, M2 = t(w1), t(m1.astype(np.uint8)), t(c2), t(m2.astype(np.uint8))
    ch, cw = m1.shape
    ws = torch.empty(blend.workspace_bytes(cw, ch) + 256, dtype=torch.uint8, device="cuda")
    pano = torch.empty((ch, cw, 3), dtype=torch.uint8, device="cuda")
    both = torch.empty((ch, cw), dtype=torch.uint8, device="cuda")
    rmse = torch.empty(1, dtype=torch.float64, device="cuda")
    eager = []
    for a, b in ((w1, c2), (w1b, c2b)):
        p, _, _, _ = blend.blend_multiband(t(a), M1, t(b), M2)
        eager.append(p.cpu().numpy())
    blend.blend_multiband(W1, M1, C2, M2, workspace=ws, pano=pano, both=both, seam_rmse=rmse)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        blend.blend_multiband(W1, M1, C2, M2, workspace=ws, pano=pano, both=both, seam_rmse=rmse,
                              stream=torch.cuda.current_stream().cuda_stream)
    for k, (a, b) in enumerate(((w1b, c2b), (w1, c2))):
        W1.copy_(t(a))
        C2.copy_(t(b))
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(pano.cpu().numpy(), eager[1 - k])
