"""Error behaviour of the drop-in surface on a host without a GPU.

The reference raises ValueError for a bad image count
(pysift/core.py:3998-4004) and a bad DSP scale count
(pysift/core.py:1203-1204); this package also raises NotImplementedError for
the learned orientation / descriptor / matcher options it does not carry,
ValueError for unknown blend and RANSAC options, and, with no CUDA device,
RuntimeError instead of falling back to a CPU path.
"""
import numpy as np
import pytest
import torch


def test_pysift_argument_errors():
    from pysift_b200 import PySIFT
    with pytest.raises(ValueError, match="dsp_n_scales"):
        PySIFT(dsp_n_scales=2)
    with pytest.raises(NotImplementedError, match="orientation"):
        PySIFT(orientation='orinet')
    with pytest.raises(NotImplementedError, match="descriptor"):
        PySIFT(descriptor='hardnet')


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour without a CUDA device")
def test_pysift_without_a_device_fails_loudly():
    from pysift_b200 import PySIFT
    with pytest.raises(RuntimeError, match="CUDA"):
        PySIFT()


@pytest.mark.parametrize("kw,exc", [
    (dict(matcher='lightglue'), NotImplementedError),
    (dict(orientation='orinet'), NotImplementedError),
    (dict(descriptor='hardnet'), NotImplementedError),
    (dict(pca_dims=32), NotImplementedError),
    (dict(blend='average'), ValueError),
    (dict(n_blend_levels=9), ValueError),
    (dict(n_blend_levels=0), ValueError),
    (dict(ransac_method='lmeds'), ValueError),
])
def test_stitcher_argument_errors(kw, exc):
    from pysift_b200 import GPUPyStitch
    with pytest.raises(exc):
        GPUPyStitch(**kw)


@pytest.mark.parametrize("n", [0, 1, 4])
def test_stitch_image_count(n):
    from pysift_b200 import GPUPyStitch
    st = GPUPyStitch.__new__(GPUPyStitch)  # the count is checked before any device state is used
    imgs = [np.zeros((8, 8, 3), np.uint8)] * n
    with pytest.raises(ValueError, match="2 or 3 images"):
        st.stitch(*imgs)
    with pytest.raises(ValueError, match="2 or 3 images"):
        st.stitch(imgs)


def test_detect_config_ranges():
    from pysift_b200 import _lib
    from pysift_b200.core import build_detect_config
    with pytest.raises(ValueError, match="n_scales"):
        build_detect_config(5, _lib.MAX_LEVELS, 1.6, 0.04, 10.0, False, 3, False, True, True, True)
    with pytest.raises(ValueError, match="n_octaves"):
        build_detect_config(_lib.MAX_OCTAVES + 1, 3, 1.6, 0.04, 10.0, False, 3, False, True, True, True)


def test_c_abi_argument_checks_without_a_device():
    """The new C entry points reject bad sizes and misaligned rows before any
    CUDA call (so these run on a host without a GPU)."""
    import ctypes
    from pysift_b200 import _lib
    lib = _lib.load()
    sz = ctypes.c_size_t()
    assert lib.pysift_pca_basis_workspace_size(128, ctypes.byref(sz)) == 0 and sz.value >= 128 * 128 * 8
    assert lib.pysift_pca_basis_workspace_size(65, ctypes.byref(sz)) == -1       # odd D
    assert lib.pysift_pca_basis_workspace_size(130, ctypes.byref(sz)) == -1      # D > 128
    fake = ctypes.c_void_p(256)  # never dereferenced: the checks fail first
    assert lib.pysift_pca_basis(fake, 64, 65, fake, 1 << 20, fake, None, None) == -1   # P > D
    assert lib.pysift_pca_basis(fake, 64, 0, fake, 1 << 20, fake, None, None) == -1    # P < 1
    assert lib.pysift_pca_basis(fake, 64, 32, fake, 16, fake, None, None) == -2        # workspace too small
    # exact uint8 matching wants 16-byte aligned rows
    odd = ctypes.c_void_p(256 + 8)
    args = (0.75, fake, 1 << 30, fake, fake, fake, fake, fake, fake, fake, None)
    assert lib.pysift_match_u8_exact(odd, 10, fake, 10, 128, *args) == -1
    assert lib.pysift_match_u8_split_fp8(fake, 10, odd, 10, 128, *args) == -1
    assert "aligned" in lib.pysift_last_error().decode()
