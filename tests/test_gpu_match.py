"""GPU parity of the tensor-core matcher against the numpy oracle."""
import numpy as np
import pytest

from pysift_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n1,n2,D", [(1000, 1000, 128), (300, 517, 128), (129, 1, 128), (1, 300, 128),
                                     (2000, 1500, 64), (8192, 8192, 128), (500, 16000, 128), (16000, 700, 128),
                                     (3001, 4099, 128)])
def test_exact_u8_bit_exact(n1, n2, D):
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import match
    a, b = synthetic.descriptor_sets(n1, n2, seed=n1 + n2, D=D)
    out = match.match_u8_exact(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    ref = mo.match_u8_exact(a, b)
    for k in ("fwd_best", "fwd_pass", "bwd_best", "bwd_pass"):
        assert np.array_equal(out[k].cpu().numpy(), ref[k]), k
    n = int(out["count"].item())
    assert np.array_equal(out["pairs"][:n].cpu().numpy(), ref["pairs"])
    assert np.array_equal(out["dist"][:n].cpu().numpy(), ref["dist"])
    if n1 >= 300 and n2 >= 300:
        assert n > 0


def test_exact_u8_ties_go_to_lower_index():
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import match
    rng = np.random.default_rng(3)
    a = rng.integers(0, 256, size=(200, 128), dtype=np.uint8)
    b = np.concatenate([a[:100], a[:100], rng.integers(0, 256, size=(60, 128), dtype=np.uint8)])
    out = match.match_u8_exact(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    ref = mo.match_u8_exact(a, b)
    assert np.array_equal(out["fwd_best"].cpu().numpy(), ref["fwd_best"])
    assert (out["fwd_best"][:100].cpu().numpy() == np.arange(100)).all()


def _unit_f16_sets(n1, n2, D, seed, dup=0):
    """Gaussian rows, L2-normalised, half of the second set noisy copies of
    the first; `dup` rows of the second set repeated exactly (fp16 ties)."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n1, D)).astype(np.float32)
    k = min(n1, n2 // 2)
    y = np.concatenate([x[:k] + 0.05 * rng.standard_normal((k, D)).astype(np.float32),
                        rng.standard_normal((n2 - k, D)).astype(np.float32)])
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y /= np.linalg.norm(y, axis=1, keepdims=True)
    xh, yh = x.astype(np.float16), y.astype(np.float16)
    if dup:  # two exact copies of the first `dup` rows at the end
        yh[n2 - 2 * dup:n2 - dup] = yh[:dup]
        yh[n2 - dup:] = yh[:dup]
    return xh, yh


def _fp16_match_and_check(xh, yh):
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import _lib, match
    out = match.match_fp16(torch.from_numpy(xh).cuda(), torch.from_numpy(yh).cuda())
    ref = mo.match_fp16(xh, yh)
    for k in ("fwd_best", "fwd_pass", "bwd_best", "bwd_pass"):
        assert np.array_equal(out[k].cpu().numpy(), ref[k]), k
    n = int(out["count"].item())
    assert np.array_equal(out["pairs"][:n].cpu().numpy(), ref["pairs"])
    assert np.array_equal(out["dist"][:n].cpu().numpy(), ref["dist"])
    # rows the candidate check could not settle went through the exact full-row pass
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")
    ws = out["workspace"]
    off = (-ws.data_ptr()) % 256
    _lib.check(_lib.load().pysift_match_fp16_recheck_counts(ws.data_ptr() + off, xh.shape[0], yh.shape[0],
                                                            xh.shape[1], cnt.data_ptr(),
                                                            torch.cuda.current_stream().cuda_stream), "counts")
    return out, ref, cnt.cpu().numpy()


@pytest.mark.parametrize("n1,n2,D", [(700, 900, 64), (1200, 800, 128), (8000, 8000, 64), (1, 300, 64),
                                     (300, 1, 64), (2, 2, 64), (3, 700, 128), (5000, 16000, 64)])
def test_fp16_reference_mode_bit_exact(n1, n2, D):
    """The stitch matcher's fp16 mode equals the oracle's exact-then-round
    similarity in every output: best indices and pass flags both ways, the
    mutual pairs and their distances."""
    xh, yh = _unit_f16_sets(n1, n2, D, seed=n1 + 7 * n2)
    out, ref, rechecked = _fp16_match_and_check(xh, yh)
    assert rechecked[0] <= n1 and rechecked[1] <= n2
    if n1 >= 300 and n2 >= 300:
        assert int(out["count"].item()) > min(n1, n2 // 2) // 2


def test_fp16_reference_mode_ties_and_rechecks():
    """Train rows 0..299 repeated twice at 900.. and 1200..: for a query whose
    best is one of them, the best, second and third similarities are equal,
    so the candidate check cannot settle the row and it is recomputed over
    every column; the lowest index wins the tie."""
    xh, yh = _unit_f16_sets(1500, 1500, 64, seed=11, dup=300)
    out, ref, rechecked = _fp16_match_and_check(xh, yh)
    fb = out["fwd_best"].cpu().numpy()
    assert (fb[:300] < 900).all()  # the copies never beat their originals
    assert rechecked[0] >= np.count_nonzero(fb[:300] == np.arange(300))


def test_fp16_reference_mode_near_ties_of_the_rounding():
    """Rows built so that the best and second similarities sit within an
    fp32 accumulation error of an fp16 rounding boundary (two train rows that
    differ in one low-order element), which a rounding of the fp32 tile
    alone can order differently from the exact similarity."""
    rng = np.random.default_rng(5)
    xh, yh = _unit_f16_sets(600, 900, 64, seed=5)
    yh = yh.copy()
    # perturb one element of a copy of each of the first 300 train rows by one fp16 ulp
    for r in range(300):
        k = int(rng.integers(64))
        v = yh[r].copy()
        v[k] = np.nextafter(v[k], np.float16(np.inf) if rng.random() < 0.5 else np.float16(-np.inf))
        yh[600 + r] = v
    _fp16_match_and_check(xh, yh)


@pytest.mark.parametrize("n1,n2,D", [(1000, 1000, 128), (300, 517, 128), (129, 1, 128), (2000, 1500, 64),
                                     (8192, 8192, 128), (500, 16000, 128)])
def test_split_fp8_bit_exact(n1, n2, D):
    """The split-nibble e4m3 GEMM gives the same exact matches as the int64 oracle."""
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import match
    a, b = synthetic.descriptor_sets(n1, n2, seed=n1 + n2 + 1, D=D)
    out = match.match_u8_split_fp8(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    ref = mo.match_u8_exact(a, b)
    for k in ("fwd_best", "fwd_pass", "bwd_best", "bwd_pass"):
        assert np.array_equal(out[k].cpu().numpy(), ref[k]), k
    n = int(out["count"].item())
    assert np.array_equal(out["pairs"][:n].cpu().numpy(), ref["pairs"])
    assert np.array_equal(out["dist"][:n].cpu().numpy(), ref["dist"])


def test_split_fp8_extreme_values_and_ties():
    """All-255 and all-0 rows, duplicates: exact distances up to 128 * 255^2."""
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import match
    rng = np.random.default_rng(9)
    a = rng.integers(0, 256, size=(300, 128), dtype=np.uint8)
    a[:10] = 255
    a[10:20] = 0
    b = np.concatenate([a[:150], a[:100], rng.integers(0, 256, size=(90, 128), dtype=np.uint8)])
    out = match.match_u8_split_fp8(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    ref = mo.match_u8_exact(a, b)
    for k in ("fwd_best", "fwd_pass", "bwd_best", "bwd_pass"):
        assert np.array_equal(out[k].cpu().numpy(), ref[k]), k


def _unit_rows(rng, n, D, dup_from=None, frac=0.5, noise=0.02):
    x = np.abs(rng.standard_normal((n, D))).astype(np.float32) if dup_from is None else None
    if dup_from is not None:
        x = rng.standard_normal((n, D)).astype(np.float32)
        k = int(frac * n)
        x[:k] = dup_from[:k] + noise * rng.standard_normal((k, D)).astype(np.float32)
    return (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)


@pytest.mark.parametrize("D", [64, 128])
def test_int8_quantisation_bit_exact(D):
    """pysift_quantize_i8_rows against the oracle and against torch's own
    expression of the reference (pysift/core.py:2902-2905)."""
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import match
    rng = np.random.default_rng(D)
    x = rng.standard_normal((3001, D)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    x[7] = 0.0  # an all-zero row: scale 127 / 1e-7
    q, s = match.quantize_i8(torch.from_numpy(x).cuda())
    rq, rs = mo.quantize_i8(x)
    assert np.array_equal(q.cpu().numpy(), rq) and np.array_equal(s.cpu().numpy(), rs)
    t = torch.from_numpy(x).cuda()
    sc = 127.0 / (t.abs().amax(dim=1, keepdim=True) + 1e-7)
    tq = (t * sc).clamp(-127, 127).to(torch.int8)
    assert torch.equal(tq, q) and torch.equal(sc[:, 0], s)


@pytest.mark.parametrize("n1,n2,D", [(1000, 1200, 64), (3000, 2500, 128), (129, 5000, 64), (8000, 8000, 64)])
def test_int8_matching_bit_exact(n1, n2, D):
    """int8 matching (tcgen05 kind::i8): every forward / backward best index,
    pass flag and mutual pair equal to the oracle's."""
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import match
    rng = np.random.default_rng(n1 + n2 + D)
    a = _unit_rows(rng, n1, D)
    b = _unit_rows(rng, n2, D, dup_from=a, frac=min(0.5, n1 / n2 * 0.5))
    q1, s1 = match.quantize_i8(torch.from_numpy(a).cuda())
    q2, s2 = match.quantize_i8(torch.from_numpy(b).cuda())
    m = match.match_i8(q1, s1, q2, s2, 0.75)
    ref = mo.match_i8(a, b, 0.75)
    for k in ("fwd_best", "fwd_pass", "bwd_best", "bwd_pass"):
        assert np.array_equal(m[k].cpu().numpy(), ref[k]), k
    n = int(m["count"].item())
    assert n == len(ref["pairs"]) and n > 0
    assert np.array_equal(m["pairs"][:n].cpu().numpy(), ref["pairs"])
    assert np.array_equal(m["dist"][:n].cpu().numpy(), ref["dist"])


def test_int8_matching_ties_go_to_lower_index():
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import match
    rng = np.random.default_rng(3)
    a = _unit_rows(rng, 300, 64)
    b = np.concatenate([a[:100], a[:100], _unit_rows(rng, 100, 64)])  # exact duplicates: equal similarities
    q1, s1 = match.quantize_i8(torch.from_numpy(a).cuda())
    q2, s2 = match.quantize_i8(torch.from_numpy(b).cuda())
    m = match.match_i8(q1, s1, q2, s2, 0.99)
    ref = mo.match_i8(a, b, 0.99)
    assert np.array_equal(m["fwd_best"].cpu().numpy(), ref["fwd_best"])
    assert np.array_equal(m["bwd_best"].cpu().numpy(), ref["bwd_best"])


def test_pca_project_f32_matches_oracle_and_fp16_path():
    import torch
    from oracle import stitch_oracle as so
    from pysift_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(11)
    x = np.abs(rng.standard_normal((2000, 128))).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    mean = x.mean(0).astype(np.float32)
    w, v = np.linalg.eigh(np.cov(x.T))
    proj = np.ascontiguousarray(v[:, -64:].astype(np.float32))
    xt, mt, pt = (torch.from_numpy(t).cuda() for t in (x, mean, proj))
    f32 = torch.empty((2000, 64), dtype=torch.float32, device="cuda")
    f16 = torch.empty((2000, 64), dtype=torch.float16, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    assert lib.pysift_pca_project_f32(xt.data_ptr(), 2000, 128, mt.data_ptr(), pt.data_ptr(), 64, f32.data_ptr(), st) == 0
    assert lib.pysift_pca_project_f16(xt.data_ptr(), 2000, 128, mt.data_ptr(), pt.data_ptr(), 64, f16.data_ptr(), st) == 0
    ref = so.pca_project(x, mean, proj)
    assert np.array_equal(f32.cpu().numpy(), ref)
    assert np.array_equal(f32.half().cpu().numpy(), f16.cpu().numpy())


def test_stitch_int8_matching_end_to_end():
    from oracle import stitch_oracle as so
    from pysift_b200.stitch import GPUPyStitch
    img1, img2, _ = synthetic.stitch_pair(480, 640, seed=6)
    st = GPUPyStitch(ransac_iters=1024, inlier_thresh=4.0, save_output=False, verbose=False, int8_matching=True)
    st.stitch(img1, img2)
    orc = so.OracleStitch(ransac_iters=1024, inlier_thresh=4.0, int8_matching=True, blend="feather").stitch(img1, img2)
    assert st.last_metrics["matches"] == len(orc["pairs"])
    assert np.array_equal(st._last["pairs"].cpu().numpy(), orc["pairs"])
    rel = np.max(np.abs(st._last["H"] - orc["H"]) / np.maximum(np.abs(orc["H"]), 1e-6))
    assert rel < 1e-6, rel
