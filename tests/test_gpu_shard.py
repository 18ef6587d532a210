"""The sharded batch API on one GPU (world size 1): the same results as the
batched call it wraps, in input order."""
import numpy as np
import pytest

from pysift_b200 import synthetic

pytestmark = pytest.mark.gpu


def test_detect_sharded_world1_equals_detect_batch():
    import torch
    from pysift_b200 import PySIFT, shard
    imgs = [synthetic.scene(h, w, seed=60 + i) for i, (h, w) in enumerate([(240, 320), (361, 479), (200, 300)])]
    sift = PySIFT()
    ref = sift.detect_batch(imgs, n_streams=2)
    got = shard.detect_sharded(sift, imgs, rank=0, world=1, n_streams=2)
    assert len(got) == len(ref)
    for (k1, d1), (k2, d2) in zip(ref, got):
        assert torch.equal(k1, k2) and torch.equal(d1, d2)
    mine = shard.detect_sharded(sift, imgs, rank=0, world=1, gather=False)
    assert sorted(mine) == [0, 1, 2]
