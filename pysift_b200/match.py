"""Brute-force ratio-test matching on the tensor cores (C ABI: pysift_match_*).

Two entry points:

* ``match_fp16(d1, d2, ratio)``: the reference's stitch-path semantics
  (pysift/core.py:2652-2701): fp16 operands, the similarity tile rounded to
  fp16, top-2 per row and per column, ratio test on d^2 = max(0, 2 - 2 s),
  mutual consistency.
* ``match_u8_exact(a, b, ratio)``: exact squared-L2 matching of uint8-valued
  descriptors through bf16 tensor-core products (exact for 128-d uint8).
* ``match_u8_split_fp8(a, b, ratio)``: the same through one e4m3 GEMM over
  split-nibble planes (v = 16 h + l).

Both take CUDA tensors and return CUDA tensors; ties go to the lower index.
"""
import ctypes

import numpy as np
import torch

from . import _lib


def _ws(lib, n1, n2, D, exact, device):
    sz = ctypes.c_size_t()
    _lib.check(lib.pysift_match_workspace_size(n1, n2, D, int(exact), ctypes.byref(sz)),
               "pysift_match_workspace_size")
    return torch.empty(int(sz.value) + 256, dtype=torch.uint8, device=device)


def _aligned(t):
    off = (-t.data_ptr()) % 256
    return t.data_ptr() + off, t.numel() - off


def _run(fn, name, d1, d2, ratio, exact, stream=None):
    lib = _lib.load()
    n1, D = d1.shape
    n2 = d2.shape[0]
    dev = d1.device
    ws = _ws(lib, n1, n2, D, exact, dev)
    wp, wn = _aligned(ws)
    out = {k: torch.empty(n, dtype=torch.int32, device=dev) for k, n in
           (("fwd_best", n1), ("fwd_pass", n1), ("bwd_best", n2), ("bwd_pass", n2))}
    pairs = torch.empty((n1, 2), dtype=torch.int32, device=dev)
    dist = torch.empty(n1, dtype=torch.float32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    st = (stream or torch.cuda.current_stream(dev)).cuda_stream
    rc = fn(d1.data_ptr(), n1, d2.data_ptr(), n2, D, float(ratio), wp, wn, out["fwd_best"].data_ptr(),
            out["fwd_pass"].data_ptr(), out["bwd_best"].data_ptr(), out["bwd_pass"].data_ptr(), pairs.data_ptr(),
            dist.data_ptr(), count.data_ptr(), st)
    _lib.check(rc, name)
    out.update(pairs=pairs, dist=dist, count=count, workspace=ws)
    return out


def match_fp16(d1, d2, ratio=0.75, stream=None):
    """d1 (N,D), d2 (M,D) float16 CUDA tensors, D in {64, 128}."""
    assert d1.dtype == torch.float16 and d2.dtype == torch.float16
    d1 = d1.contiguous()
    d2 = d2.contiguous()
    return _run(_lib.load().pysift_match_fp16, "pysift_match_fp16", d1, d2, ratio, 0, stream)


def match_u8_exact(a, b, ratio=0.75, stream=None):
    """a (N,D), b (M,D) uint8 CUDA tensors, D in {64, 128}."""
    assert a.dtype == torch.uint8 and b.dtype == torch.uint8
    return _run(_lib.load().pysift_match_u8_exact, "pysift_match_u8_exact", a.contiguous(), b.contiguous(),
                ratio, 1, stream)


def match_u8_split_fp8(a, b, ratio=0.75, stream=None):
    """The exact matching of match_u8_exact through one FP8 (e4m3) tensor-core
    GEMM over split-nibble planes: a (N,D), b (M,D) uint8 CUDA tensors."""
    assert a.dtype == torch.uint8 and b.dtype == torch.uint8
    return _run(_lib.load().pysift_match_u8_split_fp8, "pysift_match_u8_split_fp8", a.contiguous(), b.contiguous(),
                ratio, 2, stream)


def quantize_i8(x, stream=None):
    """Per-row symmetric int8 quantisation of float32 CUDA rows (N, D)
    (pysift/core.py:2902-2905): returns (int8 (N, D), float32 scales (N,))."""
    assert x.dtype == torch.float32 and x.is_cuda
    x = x.contiguous()
    n, D = x.shape
    q = torch.empty((n, D), dtype=torch.int8, device=x.device)
    s = torch.empty(n, dtype=torch.float32, device=x.device)
    st = (stream or torch.cuda.current_stream(x.device)).cuda_stream
    _lib.check(_lib.load().pysift_quantize_i8_rows(x.data_ptr(), n, D, q.data_ptr(), s.data_ptr(), st),
               "pysift_quantize_i8_rows")
    return q, s


def match_i8(q1, s1, q2, s2, ratio=0.75, stream=None):
    """int8 matching (int8_matching=True, pysift/core.py:2894-2923) of
    quantised rows q (N, D) int8 with their scales s (N,) float32, D in
    {64, 128}: similarity int32 / (s1 s2) in float32 from a tcgen05 kind::i8
    GEMM, then the fp16 mode's ratio test and mutual check."""
    assert q1.dtype == torch.int8 and q2.dtype == torch.int8
    lib = _lib.load()
    q1, q2 = q1.contiguous(), q2.contiguous()
    s1, s2 = s1.contiguous(), s2.contiguous()
    n1, D = q1.shape
    n2 = q2.shape[0]
    dev = q1.device
    ws = _ws(lib, n1, n2, D, 0, dev)
    wp, wn = _aligned(ws)
    out = {k: torch.empty(n, dtype=torch.int32, device=dev) for k, n in
           (("fwd_best", n1), ("fwd_pass", n1), ("bwd_best", n2), ("bwd_pass", n2))}
    pairs = torch.empty((n1, 2), dtype=torch.int32, device=dev)
    dist = torch.empty(n1, dtype=torch.float32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    st = (stream or torch.cuda.current_stream(dev)).cuda_stream
    rc = lib.pysift_match_i8(q1.data_ptr(), s1.data_ptr(), n1, q2.data_ptr(), s2.data_ptr(), n2, D, float(ratio),
                             wp, wn, out["fwd_best"].data_ptr(), out["fwd_pass"].data_ptr(),
                             out["bwd_best"].data_ptr(), out["bwd_pass"].data_ptr(), pairs.data_ptr(),
                             dist.data_ptr(), count.data_ptr(), st)
    _lib.check(rc, "pysift_match_i8")
    out.update(pairs=pairs, dist=dist, count=count, workspace=ws)
    return out


def to_dmatches(m):
    """The mutual matches of a match_* result as the reference's list of
    cv2.DMatch(queryIdx, trainIdx, distance) in query order
    (pysift/core.py:2929-2934), built by mapping the constructor over Python
    lists.  Reads the count, pairs and distances back to the host."""
    import cv2
    n = int(m["count"].item())
    if n == 0:
        return []
    pairs = m["pairs"][:n].cpu().numpy()
    dist = m["dist"][:n].cpu().numpy().astype(np.float64)
    return list(map(cv2.DMatch, pairs[:, 0].tolist(), pairs[:, 1].tolist(), dist.tolist()))

