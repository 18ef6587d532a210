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


@pytest.mark.parametrize("n1,n2,D", [(700, 900, 64), (1200, 800, 128)])
def test_fp16_reference_mode(n1, n2, D):
    import torch
    from oracle import match_oracle as mo
    from pysift_b200 import match
    rng = np.random.default_rng(n1)
    x = rng.standard_normal((n1, D)).astype(np.float32)
    y = np.concatenate([x[: n2 // 2] + 0.05 * rng.standard_normal((n2 // 2, D)).astype(np.float32),
                        rng.standard_normal((n2 - n2 // 2, D)).astype(np.float32)])
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y /= np.linalg.norm(y, axis=1, keepdims=True)
    xh, yh = x.astype(np.float16), y.astype(np.float16)
    out = match.match_fp16(torch.from_numpy(xh).cuda(), torch.from_numpy(yh).cuda())
    ref = mo.match_fp16(xh, yh)
    fb = out["fwd_best"].cpu().numpy()
    agree = np.mean(fb == ref["fwd_best"])
    # disagreements can only come from fp16 rounding ties of the fp32 accumulation
    assert agree >= 0.995, agree
    n = int(out["count"].item())
    assert abs(n - len(ref["pairs"])) <= max(2, 0.005 * len(ref["pairs"]))
    assert n > n2 // 4


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
