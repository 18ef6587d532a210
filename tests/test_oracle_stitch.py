"""The stitch oracle's DLT and RANSAC on the CPU.

* DLT: the oracle's homography fit against the reference's own formulation
  (pysift/core.py:2946-2981: Hartley normalisation, the 2N x 9 system, the
  last right singular vector, denormalisation, division by H[2,2]) written
  again with numpy's SVD in float64.
* RANSAC (pysift/core.py:3011-3097, MAGSAC++ and classic scores): on
  correspondences with a known homography, sub-pixel noise and planted
  outliers, the oracle recovers the homography and keeps no planted outlier.
* PCA basis (pysift/core.py:2729-2736 takes cp.linalg.eigh): the oracle's
  parallel Jacobi spans the same top-P eigenvectors as LAPACK's eigh, in the
  same order, to float32 rounding.
"""
import numpy as np
import pytest

from oracle import stitch_oracle as so
from pysift_b200 import synthetic


def _correspondences(seed, n, outliers):
    rng = np.random.default_rng(seed)
    Ht = synthetic.random_homography(rng, 1280, 960)
    p1 = np.stack([rng.uniform(0, 1280, n), rng.uniform(0, 960, n)], 1)
    ph = np.hstack([p1, np.ones((n, 1))]) @ Ht.T
    p2 = ph[:, :2] / ph[:, 2:3] + rng.normal(0, 0.7, (n, 2))
    k = int(outliers * n)
    p2[:k] = np.stack([rng.uniform(-500, 1500, k), rng.uniform(-200, 1100, k)], 1)
    return p1.astype(np.float32).astype(np.float64), p2.astype(np.float32).astype(np.float64), Ht, k


def _reference_dlt(p1, p2):
    def norm(p):
        c = p.mean(0)
        md = np.sqrt(((p - c) ** 2).sum(1)).mean()
        s = np.sqrt(2) / (md + 1e-10)
        T = np.array([[s, 0, -s * c[0]], [0, s, -s * c[1]], [0, 0, 1]], dtype=np.float64)
        return (T @ np.hstack([p, np.ones((len(p), 1))]).T).T[:, :2], T

    a, T1 = norm(p1)
    b, T2 = norm(p2)
    n = len(a)
    A = np.zeros((2 * n, 9))
    for i in range(n):
        x1, y1 = a[i]
        x2, y2 = b[i]
        A[2 * i] = [-x1, -y1, -1, 0, 0, 0, x2 * x1, x2 * y1, x2]
        A[2 * i + 1] = [0, 0, 0, -x1, -y1, -1, y2 * x1, y2 * y1, y2]
    Vt = np.linalg.svd(A, full_matrices=True)[2]
    H = np.linalg.inv(T2) @ Vt[-1].reshape(3, 3) @ T1
    return H / H[2, 2]


@pytest.mark.parametrize("seed,n", [(0, 4), (1, 5), (2, 60), (3, 400), (4, 2000)])
def test_dlt_oracle_matches_reference_svd(seed, n):
    p1, p2, _, _ = _correspondences(seed, n, 0.0)
    got = so.dlt(p1, p2)
    want = _reference_dlt(p1, p2)
    assert got[2, 2] == 1.0
    assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-9)) < 1e-6


@pytest.mark.parametrize("seed,magsac", [(10, True), (11, True), (12, False)])
def test_ransac_oracle_recovers_the_homography(seed, magsac):
    p1, p2, Ht, k = _correspondences(seed, 600, 0.3)
    H, mask, info, scores = so.ransac(p1, p2, 512, 4.0, 4.0, magsac=magsac)
    assert not mask[:k].any()
    assert mask[k:].mean() > 0.95
    assert int(info[0]) == int(mask.sum())
    corners = np.array([[0, 0, 1], [1280, 0, 1], [1280, 960, 1], [0, 960, 1]], np.float64).T
    pa, pb = H @ corners, Ht @ corners
    assert np.max(np.abs(pa[:2] / pa[2] - pb[:2] / pb[2])) < 2.0


@pytest.mark.parametrize("seed,n,D,P", [(0, 16000, 128, 64), (1, 3000, 128, 32), (2, 500, 64, 64)])
def test_pca_basis_spans_the_eigh_subspace(seed, n, D, P):
    rng = np.random.default_rng(seed)
    x = np.abs(rng.standard_normal((n, D))).astype(np.float32) ** 2
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    _, cov = so.pca_stats(x)
    basis, sweeps = so.pca_basis(cov, P, return_sweeps=True)
    assert basis.shape == (D, P) and basis.dtype == np.float32 and 0 < sweeps < 60
    w, v = np.linalg.eigh(cov)
    m = np.abs(basis.astype(np.float64).T @ v[:, -P:])
    # unit columns, orthogonal, each the eigh eigenvector of the same rank (up to sign)
    assert np.abs(np.diag(m) - 1.0).max() < 1e-6
    assert (m - np.diag(np.diag(m))).max() < 1e-5
    # and the projections the matcher uses agree to float32 rounding
    assert np.abs(x @ basis - x @ v[:, -P:].astype(np.float32) * np.sign(np.diag(basis.T @ v[:, -P:]))).max() < 1e-5
