"""Build recipe: the reference's own CUDA kernels as a shared library --
TEST INFRASTRUCTURE ONLY.

    python oracle/build_ref.py [/path/to/reference]

pysift/core.py of the reference (SivaIITM/PySIFT) carries its hot-path
kernels as CUDA C source strings handed to cp.RawKernel: find_extrema_fused
(core.py:176-217), orientation_hist (228-333), refine_keypoints (343-463,
compiled there with --use_fast_math), gauss_h / gauss_v (475-547) and
sift_descriptor_coop (693-835).  This recipe reads those strings out of
the reference's source with `ast` (nothing of the reference is imported or
run), writes each to its own translation unit in a temporary directory
outside this repository, and compiles them with nvcc for sm_100a, with the
options CuPy's NVRTC build uses (default optimisation, FMA contraction on;
--use_fast_math for refine_keypoints only), together with
oracle/ref_shim.cu (launchers with the reference's grid and block shapes)
into oracle/_ref/libpysift_ref_kernels.so.  tests/ref_runner.py drives them
to pin the product against the reference's own kernels on the GPU.

The reference checkout is taken from the argument, else from
PYSIFT_REFERENCE, else /root/reference.  Without it nothing is built.
"""
import ast
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libpysift_ref_kernels.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# kernel name -> (variable holding the RawKernel, extra options)
KERNELS = {
    "find_extrema_fused": [],
    "orientation_hist": [],
    "refine_keypoints": ["--use_fast_math"],
    "gauss_h": [],
    "gauss_v": [],
    "sift_descriptor_coop": [],
}


def reference_root(argv):
    if len(argv) > 1:
        return argv[1]
    return os.environ.get("PYSIFT_REFERENCE") or "/root/reference"


def kernel_sources(core_py):
    """{kernel name: CUDA source} of every cp.RawKernel(src, name, ...) in the file."""
    tree = ast.parse(open(core_py).read())
    strings = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and isinstance(node.value, ast.Constant) and isinstance(node.value.value, str):
            for t in node.targets:
                if isinstance(t, ast.Name):
                    strings[t.id] = node.value.value
    out = {}
    for node in ast.walk(tree):
        if not (isinstance(node, ast.Call) and isinstance(node.func, ast.Attribute) and node.func.attr == "RawKernel"):
            continue
        if len(node.args) < 2 or not isinstance(node.args[1], ast.Constant):
            continue
        src = node.args[0]
        if isinstance(src, ast.Constant):
            code = src.value
        elif isinstance(src, ast.Name) and src.id in strings:
            code = strings[src.id]
        else:
            continue
        out[node.args[1].value] = code
    return out


def build(argv=sys.argv):
    root = reference_root(argv)
    core_py = os.path.join(root, "pysift", "core.py")
    if not os.path.isfile(core_py):
        print(f"build_ref: no reference checkout at {root}; nothing built")
        return None
    srcs = kernel_sources(core_py)
    missing = [k for k in KERNELS if k not in srcs]
    if missing:
        raise RuntimeError(f"build_ref: kernels not found in {core_py}: {missing}")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    os.makedirs(OUT_DIR, exist_ok=True)
    with tempfile.TemporaryDirectory(prefix="pysift_ref_") as tmp:
        objs = []
        for name, opts in KERNELS.items():
            cu = os.path.join(tmp, name + ".cu")
            with open(cu, "w") as f:
                f.write(srcs[name])
            obj = os.path.join(tmp, name + ".o")
            subprocess.check_call([nvcc, *ARCH, "-O3", *opts, "-Xcompiler", "-fPIC", "-c", cu, "-o", obj])
            objs.append(obj)
        shim = os.path.join(tmp, "ref_shim.o")
        subprocess.check_call([nvcc, *ARCH, "-O3", "-Xcompiler", "-fPIC", "-c", os.path.join(HERE, "ref_shim.cu"),
                               "-o", shim])
        tmp_lib = LIB + ".tmp"
        subprocess.check_call([nvcc, *ARCH, "-shared", "-o", tmp_lib, *objs, shim])
        os.replace(tmp_lib, LIB)
    print("built", LIB)
    return LIB


if __name__ == "__main__":
    build()
