"""The blur tile-height autotuner's host side on the CPU: the levels a
detection blurs, the library's size classes and table checks, and the JSON
cache round trip (no device work)."""
import types

import numpy as np
import pytest


def test_pyramid_levels_of_the_default_configuration():
    from pysift_b200 import autotune
    from pysift_b200.core import build_detect_config
    cfg = build_detect_config(5, 3, 1.6, 0.04, 10.0, False, 3, False, True, True, True)
    levels = autotune.pyramid_levels(types.SimpleNamespace(_cfg=cfg), 480, 640)
    assert levels[0] == (5, 960, 1280)  # base blur of the doubled image
    assert len(levels) == 1 + 5 * 5
    assert [R for R, _, _ in levels[1:6]] == [5, 6, 8, 10, 12]
    assert levels[6][1:] == (480, 640) and levels[-1][1:] == (60, 80)


def test_size_classes_and_table_checks():
    from pysift_b200 import _lib
    lib = _lib.load()
    assert lib.pysift_blur_size_class(32, 32) == 0
    assert lib.pysift_blur_size_class(1, 1) == 0
    assert lib.pysift_blur_size_class(960, 1280) == 20 - 10
    assert lib.pysift_blur_size_class(1 << 14, 1 << 14) == 15
    assert lib.pysift_blur_size_class(0, 5) == -1
    t = np.zeros(17 * 16, np.int32)
    assert lib.pysift_set_blur_tile_table(t.ctypes.data, t.size) == 0
    assert lib.pysift_set_blur_tile_table(t.ctypes.data, 5) != 0
    t[5 * 16 + 10] = 24
    assert lib.pysift_set_blur_tile_table(t.ctypes.data, t.size) != 0
    t[5 * 16 + 10] = 40
    assert lib.pysift_set_blur_tile_table(t.ctypes.data, t.size) == 0
    assert lib.pysift_set_blur_tile_table(None, 0) == 0


def test_cache_round_trip(tmp_path):
    from pysift_b200 import autotune
    best = {(5, 10): 40, (12, 10): 32, (6, 8): 16}
    p = tmp_path / "t" / "blur.json"
    autotune.save(best, str(p))
    assert autotune.load(str(p)) == best
    table = autotune.to_table(best)
    assert table.shape == (17 * 16,) and table[5 * 16 + 10] == 40 and table[6 * 16 + 8] == 16
    assert np.count_nonzero(table) == 3
