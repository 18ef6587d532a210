"""Regenerates tests/golden/imc_st_pauls_*.{png,npz} from the reference tree.

The reference (SivaIITM/PySIFT) ships golden detectAndCompute dumps in
determinism_reference/ (made on an RTX 3050 with n_octaves=4, DSP-5,
fp16 pyramid -- determinism_reference/manifest.json).  This keeps a compact
copy of one of them: the decoded grayscale source image (lossless PNG), all
keypoint rows (points, angles, sizes) and every 16th descriptor row.

    python tests/golden/make_golden.py /path/to/reference
    (or with the path in PYSIFT_REFERENCE)
"""
import os
import sys

import cv2
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    name = "imc_st_pauls_cathedral"
    src = os.path.join(ref_root, "test_images", "imc_phototourism", "st_pauls_cathedral",
                       "21260922_4094863925.jpg")
    gray = cv2.imread(src, cv2.IMREAD_GRAYSCALE)
    fx = np.load(os.path.join(ref_root, "determinism_reference", name + ".npz"))
    assert tuple(fx["image_shape"][:2]) == gray.shape
    cv2.imwrite(os.path.join(HERE, name + "_gray.png"), gray, [cv2.IMWRITE_PNG_COMPRESSION, 9])
    rows = np.arange(0, len(fx["points"]), 16)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), points=fx["points"], angles=fx["angles"],
                        sizes=fx["sizes"], desc_rows=rows, descriptors=fx["descriptors"][rows],
                        image_shape=fx["image_shape"])


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYSIFT_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py /path/to/reference (or set PYSIFT_REFERENCE)")
    main(root)
