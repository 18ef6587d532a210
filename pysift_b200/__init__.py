"""pysift_b200 -- B200-native SIFT-and-stitching hot path with PySIFT's API.

``from pysift_b200 import PySIFT, GPUPyStitch`` gives drop-in classes for the
reference's ``pysift.PySIFT`` and ``pysift.GPUPyStitch`` (SivaIITM/PySIFT,
pysift/__init__.py:5-7).  The GPU work runs in hand-written sm_100a CUDA
kernels in libpysift_b200.so, called through the C ABI declared in
include/pysift_b200.h.
"""
__version__ = "0.1.0"

from .core import PySIFT  # noqa: E402
from .stitch import GPUPyStitch  # noqa: E402

__all__ = ["PySIFT", "GPUPyStitch"]
