"""CPU oracle for ratio-test matching -- TEST INFRASTRUCTURE ONLY.

Restates pysift/core.py:2652-2701 (_match_symmetric) and 2840-2940
(_match_features' mutual intersection) in numpy, with the canonical
tie-break (equal scores: lower index first) that the reference leaves to
torch.topk.

* fp16 mode: the similarity is the fp16 rounding of the EXACT dot product
  of the fp16 operands (float64 accumulation is exact for D <= 128 here up
  to one final rounding); the GPU's fp32 tensor-core accumulation can
  differ from it only when the exact value lies within ~1e-7 of an fp16
  rounding boundary.
* exact mode: int64 squared L2 distances of uint8 descriptors.
* int8 mode (int8_matching=True, pysift/core.py:2894-2923): per-row
  symmetric quantisation of the float32 (PCA-projected, L2-normalised)
  descriptors, an exact int32 GEMM, the similarity int / (s1 s2) in float32,
  then the fp16 mode's ratio test on it.
"""
import numpy as np


def _top2(keys, larger_is_better):
    """Per-row (best idx, best key, second key) with lower-index ties:
    np.argmax/argmin return the first extremum, and the second key is the
    extremum of the row with the winner masked out."""
    n, m = keys.shape
    rows = np.arange(n)
    b1 = np.argmax(keys, axis=1) if larger_is_better else np.argmin(keys, axis=1)
    k1 = keys[rows, b1]
    if m < 2:
        return b1, k1, np.full(n, np.nan)
    masked = keys.copy()
    if np.issubdtype(keys.dtype, np.floating):
        masked[rows, b1] = -np.inf if larger_is_better else np.inf
    else:
        info = np.iinfo(keys.dtype)
        masked[rows, b1] = info.min if larger_is_better else info.max
    k2 = masked.max(axis=1) if larger_is_better else masked.min(axis=1)
    return b1, k1, k2


def sim_fp16(d1h, d2h):
    a = d1h.astype(np.float64)
    b = d2h.astype(np.float64)
    return (a @ b.T).astype(np.float16).astype(np.float32)


def ratio_pass_fp16(s1, s2, ratio_sq=np.float32(0.5625)):
    db = np.maximum(np.float32(2.0) - np.float32(2.0) * s1, np.float32(0.0))
    ds = np.maximum(np.float32(2.0) - np.float32(2.0) * s2, np.float32(0.0))
    ok = (ds > np.float32(1e-10)) & (db < ratio_sq * ds)
    return ok, np.sqrt(db)


def match_fp16(d1h, d2h, ratio=0.75):
    S = sim_fp16(d1h, d2h)
    rs = np.float32(ratio * ratio)
    fb, f1, f2 = _top2(S, True)
    fok, fdist = ratio_pass_fp16(f1, f2, rs)
    bb, b1, b2 = _top2(S.T.copy(), True)
    bok, _ = ratio_pass_fp16(b1, b2, rs)
    return _mutual(fb, fok, fdist, bb, bok, S)


def match_u8_exact(a, b, ratio=0.75):
    A = a.astype(np.int64)
    B = b.astype(np.int64)
    # float64 products and sums of uint8 values are exact integers (< 2^53)
    G = (a.astype(np.float64) @ b.astype(np.float64).T).astype(np.int64)
    D2 = (A * A).sum(1)[:, None] + (B * B).sum(1)[None, :] - 2 * G
    rs = ratio * ratio
    fb, f1, f2 = _top2(D2, False)
    fok = (f2 > 0) & (f1.astype(np.float64) < rs * f2.astype(np.float64))
    bb, b1, b2 = _top2(D2.T.copy(), False)
    bok = (b2 > 0) & (b1.astype(np.float64) < rs * b2.astype(np.float64))
    return _mutual(fb, fok, np.sqrt(f1.astype(np.float32)), bb, bok, D2)


def _mutual(fb, fok, fdist, bb, bok, S):
    pairs = []
    dist = []
    for i in range(len(fb)):
        if fok[i]:
            j = int(fb[i])
            if bok[j] and bb[j] == i:
                pairs.append((i, j))
                dist.append(fdist[i])
    return dict(fwd_best=fb.astype(np.int32), fwd_pass=fok.astype(np.int32), bwd_best=bb.astype(np.int32),
                bwd_pass=bok.astype(np.int32), pairs=np.array(pairs, np.int32).reshape(-1, 2),
                dist=np.array(dist, np.float32), scores=S)


def quantize_i8(d):
    """_to_int8_torch (pysift/core.py:2902-2905) in float32: scale =
    127.0 / (max |d| + 1e-7) per row, which torch evaluates (scalar / tensor)
    as reciprocal(max |d| + 1e-7) * 127; q = trunc(clip(d * scale, -127, 127))."""
    d = np.asarray(d, np.float32)
    scale = (np.float32(1.0) / (np.abs(d).max(axis=1) + np.float32(1e-7))) * np.float32(127.0)
    q = np.trunc(np.clip(d * scale[:, None], np.float32(-127.0), np.float32(127.0))).astype(np.int8)
    return q, scale.astype(np.float32)


def sim_i8(q1, s1, q2, s2):
    """torch._int_mm(q1, q2.T).float() / (s1 * s2.T) (pysift/core.py:2908-2910)."""
    acc = q1.astype(np.int64) @ q2.astype(np.int64).T
    den = s1[:, None].astype(np.float32) * s2[None, :].astype(np.float32)
    return acc.astype(np.float32) / den


def match_i8(d1, d2, ratio=0.75):
    """int8 matching of float32 descriptors (quantised here)."""
    q1, s1 = quantize_i8(d1)
    q2, s2 = quantize_i8(d2)
    S = sim_i8(q1, s1, q2, s2)
    rs = np.float32(ratio * ratio)
    fb, f1, f2 = _top2(S, True)
    fok, fdist = ratio_pass_fp16(f1, f2, rs)
    bb, b1, b2 = _top2(S.T.copy(), True)
    bok, _ = ratio_pass_fp16(b1, b2, rs)
    out = _mutual(fb, fok, fdist, bb, bok, S)
    out.update(q1=q1, s1=s1, q2=q2, s2=s2)
    return out

