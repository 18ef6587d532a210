"""Build recipe for the sm_100a shared library (in-tree, no JIT cache).

    python -m pysift_b200.build

compiles pysift_b200/csrc/*.cu with nvcc for sm_100a into
pysift_b200/libpysift_b200.so.  --fmad=false makes every floating-point
operator a single IEEE operation (the kernels spell out their fused
multiply-adds with fmaf), which is what lets a CPU restatement reproduce
their results bit for bit.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpysift_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def build(verbose=False, force=False):
    srcs = sources()
    deps = srcs + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    if not force and os.path.exists(LIB_PATH):
        lib_m = os.path.getmtime(LIB_PATH)
        if all(os.path.getmtime(d) <= lib_m for d in deps):
            return LIB_PATH
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", "-o", tmp, *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
