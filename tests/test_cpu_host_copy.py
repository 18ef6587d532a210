"""pysift_host_copy (the threaded staging copy of host images, a host
function of the C library): byte-exact for sizes around the 1 MiB threshold
and the page-sized pieces, for every thread count, and from several Python
threads at once; argument checks."""
import threading

import numpy as np
import pytest


@pytest.mark.parametrize("n", [0, 1, 4095, (1 << 20) - 1, 1 << 20, (1 << 20) + 4097, 3_686_400, 7_000_001])
@pytest.mark.parametrize("threads", [1, 2, 4, 8, 64])
def test_host_copy_is_byte_exact(n, threads):
    from pysift_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(n + threads)
    src = rng.integers(0, 256, size=n + 64, dtype=np.uint8)
    dst = np.zeros(n + 64, dtype=np.uint8)
    # odd offsets on both sides
    assert lib.pysift_host_copy(dst.ctypes.data + 3, src.ctypes.data + 5, n, threads) == 0
    assert np.array_equal(dst[3:3 + n], src[5:5 + n])
    assert not dst[:3].any() and not dst[3 + n:].any()


def test_host_copy_from_concurrent_callers():
    from pysift_b200 import _lib
    lib = _lib.load()
    n = 5_000_000
    srcs = [np.full(n, i + 1, dtype=np.uint8) for i in range(6)]
    dsts = [np.zeros(n, dtype=np.uint8) for _ in range(6)]
    errs = []

    def work(i):
        for _ in range(5):
            if lib.pysift_host_copy(dsts[i].ctypes.data, srcs[i].ctypes.data, n, 4) != 0:
                errs.append(i)

    ts = [threading.Thread(target=work, args=(i,)) for i in range(6)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=60)
    assert not errs and all(np.array_equal(d, s) for d, s in zip(dsts, srcs))


def test_host_copy_argument_checks():
    from pysift_b200 import _lib
    lib = _lib.load()
    buf = np.zeros(16, dtype=np.uint8)
    assert lib.pysift_host_copy(None, buf.ctypes.data, 16, 4) == -1
    assert lib.pysift_host_copy(buf.ctypes.data, buf.ctypes.data, 16, 0) == -1
    assert lib.pysift_host_copy(buf.ctypes.data, buf.ctypes.data, 16, 65) == -1
    assert lib.pysift_host_copy(None, None, 0, 4) == 0
