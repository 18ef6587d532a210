"""The matching oracle against independent restatements, on the CPU.

* fp16 mode: the reference's `_match_symmetric` (pysift/core.py:2652-2701)
  and mutual intersection (pysift/core.py:2934-2940) written again with
  torch.topk on the CPU, over the same fp16 similarity matrix.  A row whose
  best score is tied fails the ratio test (d_best < 0.5625 d_second is false
  for d_best == d_second), so the pass flags and the mutual pairs do not
  depend on how topk orders ties and are compared exactly.
* int8 mode: the reference's `_to_int8_torch` and rescale
  (pysift/core.py:2896-2904) run as written, in torch float32 on the CPU,
  against the oracle's quantisation and similarity, bit for bit.
* exact mode: squared L2 of uint8 descriptors by plain Python loops, with
  planted duplicate rows so that the best and second-best ties occur; the
  oracle keeps the lower index.
"""
import numpy as np
import torch

from oracle import match_oracle as mo


def _desc_pair(n, m, d, seed):
    rng = np.random.default_rng(seed)
    a = np.abs(rng.standard_normal((n, d))).astype(np.float32)
    b = np.abs(rng.standard_normal((m, d))).astype(np.float32)
    k = min(n, m) // 2
    b[:k] = a[:k] + 0.15 * np.abs(rng.standard_normal((k, d))).astype(np.float32)
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b /= np.linalg.norm(b, axis=1, keepdims=True)
    return a, b


def _reference_symmetric(sim_f, ratio):
    """Forward / backward dicts {i: (j, dist)} as pysift/core.py:2676-2700 builds them."""
    ratio_sq = ratio ** 2
    out = []
    for s in (sim_f, sim_f.T):
        v, idx = torch.topk(s, k=2, dim=1, largest=True, sorted=True)
        d_best = torch.clamp(2.0 - 2.0 * v[:, 0], min=0.0)
        d_second = torch.clamp(2.0 - 2.0 * v[:, 1], min=0.0)
        ok = ((d_second > 1e-10) & (d_best < ratio_sq * d_second)).numpy()
        j = idx[:, 0].numpy().astype(np.int32)
        dist = torch.sqrt(d_best).numpy().astype(np.float32)
        out.append({i: (int(j[i]), float(dist[i])) for i in range(s.shape[0]) if ok[i]})
    return out


def _mutual(fwd, bwd):
    return [(i, j, d) for i, (j, d) in fwd.items() if j in bwd and bwd[j][0] == i]


def test_fp16_oracle_matches_reference_symmetric():
    for seed, (n, m) in enumerate([(300, 257), (64, 500), (2, 3)]):
        a, b = _desc_pair(n, m, 64, seed)
        ah, bh = a.astype(np.float16), b.astype(np.float16)
        got = mo.match_fp16(ah, bh, 0.75)
        sim_f = torch.from_numpy(mo.sim_fp16(ah, bh))
        fwd, bwd = _reference_symmetric(sim_f, 0.75)
        assert sorted(fwd) == np.flatnonzero(got["fwd_pass"]).tolist()
        assert sorted(bwd) == np.flatnonzero(got["bwd_pass"]).tolist()
        want = _mutual(fwd, bwd)
        assert got["pairs"].tolist() == [[i, j] for i, j, _ in want]
        assert got["dist"].tolist() == [np.float32(d).item() for _, _, d in want]
        if n >= 64:
            assert len(want) > 10


def test_int8_oracle_matches_reference_expressions():
    a, b = _desc_pair(200, 180, 64, 7)
    a[3] = 0.0  # an all-zero row: scale 127 / 1e-7
    got = mo.match_i8(a, b, 0.75)

    def to_int8(d):
        d_t = torch.from_numpy(d)
        scale = 127.0 / (d_t.abs().amax(dim=1, keepdim=True) + 1e-7)
        return (d_t * scale).clamp(-127, 127).to(torch.int8), scale

    q1, s1 = to_int8(a)
    q2, s2 = to_int8(b)
    assert np.array_equal(q1.numpy(), got["q1"]) and np.array_equal(q2.numpy(), got["q2"])
    assert np.array_equal(s1.numpy()[:, 0].view(np.int32), got["s1"].view(np.int32))
    sim_i32 = (q1.long() @ q2.long().T).to(torch.int32)
    sim_f32 = sim_i32.float() / (s1 * s2.T)
    assert np.array_equal(sim_f32.numpy().view(np.int32), got["scores"].view(np.int32))
    fwd, bwd = _reference_symmetric(sim_f32, 0.75)
    assert got["pairs"].tolist() == [[i, j] for i, j, _ in _mutual(fwd, bwd)]


def test_exact_u8_oracle_against_loops_with_ties():
    rng = np.random.default_rng(11)
    n, m, d = 23, 31, 16
    a = rng.integers(0, 256, (n, d), dtype=np.uint8)
    b = rng.integers(0, 256, (m, d), dtype=np.uint8)
    b[5] = a[2]
    b[9] = a[2]          # exact best tie for query 2: lower index 5 wins, and the row fails the ratio test
    b[12] = a[4]
    b[20] = np.clip(a[4].astype(int) + 1, 0, 255).astype(np.uint8)
    b[27] = b[20]        # tied second best for query 4
    got = mo.match_u8_exact(a, b, 0.75)
    D2 = [[sum((int(a[i, k]) - int(b[j, k])) ** 2 for k in range(d)) for j in range(m)] for i in range(n)]

    def best2(rows):
        out = []
        for r in rows:
            j1 = min(range(len(r)), key=lambda j: (r[j], j))
            second = min(r[j] for j in range(len(r)) if j != j1)
            out.append((j1, r[j1], second))
        return out

    fw = best2(D2)
    bw = best2([list(col) for col in zip(*D2)])
    assert got["fwd_best"].tolist() == [t[0] for t in fw]
    assert got["bwd_best"].tolist() == [t[0] for t in bw]
    fok = [t[2] > 0 and t[1] < 0.5625 * t[2] for t in fw]
    bok = [t[2] > 0 and t[1] < 0.5625 * t[2] for t in bw]
    assert got["fwd_pass"].tolist() == [int(x) for x in fok]
    assert got["bwd_pass"].tolist() == [int(x) for x in bok]
    assert fw[2][0] == 5 and not fok[2]
    assert fok[4] and fw[4][0] == 12
    want = [[i, fw[i][0]] for i in range(n) if fok[i] and bok[fw[i][0]] and bw[fw[i][0]][0] == i]
    assert got["pairs"].tolist() == want and [4, 12] in want
    assert np.array_equal(got["dist"], np.sqrt(np.array([fw[i][1] for i, _ in want], np.float32)))
