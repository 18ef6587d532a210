"""Gradients of the differentiable descriptor and warp + feather blend:
hand-written CUDA backward against a plain torch-autograd restatement
(float64) and against float64 central finite differences on 64x64 crops."""
import numpy as np
import pytest

from pysift_b200 import synthetic

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def _img(H, W, seed):
    """A smooth random texture with no flat region: the descriptor's
    |gradient| has a cone point where the level is flat, and there neither the
    orientation nor the gradient of the descriptor is defined."""
    import cv2
    rng = np.random.default_rng(seed)
    t = cv2.GaussianBlur(rng.standard_normal((H, W)), (0, 0), 2.0)
    yy, xx = np.mgrid[0:H, 0:W]
    t = t / (t.std() + 1e-12) + 0.3 * np.sin(xx / 7.0) + 0.2 * np.cos(yy / 5.0)
    t = (t - t.min()) / (t.max() - t.min())
    return (0.1 + 0.8 * t).astype(np.float32)


def _sift(n_oct=2):
    from pysift_b200 import PySIFT
    return PySIFT(double_image=False, n_octaves=n_oct)


def _kps(rng, H, W, n, octaves=(0,), ph_max=34):
    rows = []
    for _ in range(n):
        o = int(rng.choice(octaves))
        si = int(rng.integers(1, 4))
        h, w = H >> o, W >> o
        rows.append([o, si, rng.integers(2, h - 2), rng.integers(2, w - 2), rng.uniform(0, 360)])
    import torch
    return torch.tensor(np.array(rows, np.float64))


def test_blur_adjoint_is_the_transpose():
    import torch
    from pysift_b200 import grad
    from pysift_b200.core import gaussian_weights
    rng = np.random.default_rng(0)
    for (H, W, sigma) in [(57, 83, 1.2), (128, 96, 3.0), (40, 40, 2.2)]:
        w, r = gaussian_weights(sigma)
        x = torch.from_numpy(rng.standard_normal((H, W)).astype(np.float32)).cuda()
        y = torch.from_numpy(rng.standard_normal((H, W)).astype(np.float32)).cuda()
        bx = grad._blur(x, w, r)
        bty = grad._blur_adjoint(y, w, r)
        lhs = float((bx.double() * y.double()).sum())
        rhs = float((x.double() * bty.double()).sum())
        assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), 1.0)


def test_descriptor_forward_and_grad_match_torch_autograd():
    import torch
    from pysift_b200 import grad
    rng = np.random.default_rng(1)
    H, W = 160, 200
    sift = _sift(2)
    img = torch.from_numpy(_img(H, W, 3)).cuda()
    kps = _kps(rng, H, W, 24, octaves=(0, 0, 1))
    x = img.clone().requires_grad_(True)
    d = grad.descriptors(x, kps, sift)
    r = torch.from_numpy(rng.standard_normal(d.shape).astype(np.float32)).cuda()
    (d * r).sum().backward()
    x64 = img.double().clone().requires_grad_(True)
    d64 = grad.descriptors_torch(x64, kps, sift)
    (d64 * r.double()).sum().backward()
    assert _rel(d.detach().cpu(), d64.detach().cpu()) < 1e-4
    assert _rel(x.grad.cpu(), x64.grad.cpu()) < 1e-4


def test_descriptor_grad_finite_differences_64x64():
    import torch
    from pysift_b200 import grad
    rng = np.random.default_rng(2)
    sift = _sift(1)
    img = torch.from_numpy(_img(64, 64, 4)).cuda()
    kps = torch.tensor([[0, 1, 32, 31, 17.0], [0, 1, 30, 34, 200.0], [0, 2, 33, 32, 95.0]], dtype=torch.float64)
    r = torch.from_numpy(rng.standard_normal((3, 128))).cuda()

    def loss64(z):
        return (grad.descriptors_torch(z, kps, sift) * r).sum()

    x = img.clone().requires_grad_(True)
    (grad.descriptors(x, kps, sift) * r.float()).sum().backward()
    g_cuda = x.grad.double()
    x64 = img.double().clone().requires_grad_(True)
    loss64(x64).backward()
    g_ref = x64.grad
    assert _rel(g_cuda.cpu(), g_ref.cpu()) < 1e-4
    eps = 1e-6
    for _ in range(6):
        v = torch.from_numpy(rng.standard_normal((64, 64))).cuda()
        with torch.no_grad():
            fd = float((loss64(img.double() + eps * v) - loss64(img.double() - eps * v)) / (2 * eps))
        # the size of a random directional derivative: |g| |v| / sqrt(N)
        scale = float(g_ref.norm() * v.norm()) / 64.0
        assert abs(fd - float((g_ref * v).sum())) <= 1e-4 * scale
        assert abs(fd - float((g_cuda * v).sum())) <= 1e-4 * scale


def _warp_case(seed, H=48, W=64):
    import torch
    from pysift_b200 import grad
    rng = np.random.default_rng(seed)
    a = rng.random((H, W, 3))
    b = rng.random((H, W, 3))
    Hm = synthetic.random_homography(rng, W, H)
    Hm[0, 2] *= 0.5  # keep a wide overlap on these small views
    geo = grad.canvas_geometry(a.shape, b.shape, Hm)
    h8 = torch.from_numpy(Hm.ravel()[:8].copy())
    return torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), h8.cuda(), geo, rng


def test_warp_blend_forward_and_grads_match_torch_autograd():
    import torch
    from pysift_b200 import grad
    a, b, h8, geo, rng = _warp_case(5)
    x1 = a.float().clone().requires_grad_(True)
    x2 = b.float().clone().requires_grad_(True)
    hh = h8.clone().requires_grad_(True)
    out = grad.warp_blend(x1, x2, hh, geo)
    tgt = torch.from_numpy(rng.random(tuple(out.shape))).cuda()
    ((out.double() - tgt) ** 2).sum().backward()
    y1 = a.clone().requires_grad_(True)
    y2 = b.clone().requires_grad_(True)
    h64 = h8.clone().requires_grad_(True)
    ref = grad.warp_blend_torch(y1, y2, h64, geo)
    ((ref - tgt) ** 2).sum().backward()
    assert _rel(out.detach().cpu(), ref.detach().cpu()) < 1e-5
    assert _rel(x1.grad.cpu(), y1.grad.cpu()) < 1e-4
    assert _rel(x2.grad.cpu(), y2.grad.cpu()) < 1e-4
    assert _rel(hh.grad.cpu(), h64.grad.cpu()) < 1e-4


def test_warp_blend_homography_grad_finite_differences():
    import torch
    from pysift_b200 import grad
    a, b, h8, geo, rng = _warp_case(6, 64, 64)
    tgt = torch.from_numpy(rng.random((geo[1], geo[0], 3))).cuda()

    def loss64(h):
        return ((grad.warp_blend_torch(a, b, h, geo) - tgt) ** 2).sum()

    hh = h8.clone().requires_grad_(True)
    ((grad.warp_blend(a.float(), b.float(), hh, geo).double() - tgt) ** 2).sum().backward()
    h64 = h8.clone().requires_grad_(True)
    loss64(h64).backward()
    assert _rel(hh.grad.cpu(), h64.grad.cpu()) < 1e-4
    scale = np.abs(h8.cpu().numpy()) + 1e-3
    for k in range(8):
        e = torch.zeros(8, dtype=torch.float64, device="cuda")
        e[k] = 1e-6 * scale[k]
        with torch.no_grad():
            fd = (loss64(h8 + e) - loss64(h8 - e)) / (2 * e[k])
        assert abs(float(fd) - float(h64.grad[k])) <= 1e-4 * max(abs(float(h64.grad[k])), 1e-6) + 1e-3
