"""The blur tile-height autotuner on the GPU: it measures every height for
the levels a detection blurs, caches the winners per GPU, and a detection
with the tuned table is still bit-exact against the oracle."""
import numpy as np
import pytest

from pysift_b200 import synthetic

pytestmark = pytest.mark.gpu


def test_autotuned_detection_unchanged(tmp_path, oracle_lib):
    from pysift_b200 import PySIFT, autotune
    sift = PySIFT()
    path = str(tmp_path / "blur_tiles.json")
    try:
        best = sift.autotune(480, 640, path=path)
        assert len(best) >= 5 and set(best.values()) <= {16, 32, 40}
        assert autotune.load(path) == best
        img = synthetic.scene(480, 640, seed=5)
        out = sift.detect_arrays(img)
        ref = oracle_lib.OracleSIFT().detect_and_compute(img)
        for k in ("x", "y", "size", "angle", "response", "octave", "desc"):
            assert np.array_equal(out[k], ref[k]), k
        # a second call finds every entry in the cache and measures nothing new
        assert sift.autotune(480, 640, path=path) == best
    finally:
        autotune.clear()
