"""Regenerate the golden fixtures under tests/golden/ from a chfem source tree.

The reference's own regression data (its test/input/3D directory: two voxel images, their
.nf settings files and the golden effective-tensor columns; test/input/2D: a pixel image and
the golden thermal, elastic and permeability tensors) is copied here so that the parity tests can run where
the reference tree is absent.  Images are stored gzip-compressed.

Usage:  python tests/golden/make_fixtures.py [/path/to/chfem]
"""
import gzip
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # name: (image, shape z,y,x, nf file, result file, golden column, reference tolerance)
    "thermal_ggg40": ("3D/ggg40_100.raw", (100, 100, 100), "3D/thermal/ggg40_100.nf",
                      "3D/thermal/ggg40_100_result.bin", 0),
    "elastic_ggg40": ("3D/ggg40_100.raw", (100, 100, 100), "3D/elastic/ggg40_100.nf",
                      "3D/elastic/ggg40_100_result.bin", 1),
    "fluid_fibers": ("3D/fibers_100x100x10.raw", (10, 100, 100), "3D/fluid/fibers_100x100x10.nf",
                     "3D/fluid/fibers_100x100x10_result.bin", 2),
}
# 2D cases: the whole tensor (every load case), thermal 2 x 2 and elastic 3 x 3
CASES_2D = {
    "thermal_2d": ("2D/100x100.raw", (100, 100), "2D/thermal/100x100.nf", "2D/thermal/100x100_result.bin", 2),
    "elastic_2d": ("2D/100x100.raw", (100, 100), "2D/elastic/100x100.nf", "2D/elastic/100x100_result.bin", 3),
    "fluid_2d": ("2D/100x100.raw", (100, 100), "2D/fluid/100x100.nf", "2D/fluid/100x100_result.bin", 2),
}


def main(ref_root):
    src = os.path.join(ref_root, "test", "input")
    manifest = {}
    for name, (img, shape, nf, res, col) in CASES.items():
        img_out = os.path.join(HERE, os.path.basename(img) + ".gz")
        if not os.path.exists(img_out):
            with open(os.path.join(src, img), "rb") as fi, gzip.open(img_out, "wb", compresslevel=9) as fo:
                shutil.copyfileobj(fi, fo)
        nf_out = name + ".nf"
        shutil.copyfile(os.path.join(src, nf), os.path.join(HERE, nf_out))
        vals = np.fromfile(os.path.join(src, res), dtype=np.float64)
        k = 6 if name.startswith("elastic") else 3
        C = vals[: k * k].reshape(k, k)
        manifest[name] = {
            "image": os.path.basename(img_out),
            "shape_zyx": list(shape),
            "nf": nf_out,
            "direction": col,
            "column": [float(v) for v in C[:, col]],
            "reference_tolerance": 1e-4,
            "source": f"test/input/{res}",
        }
    for name, (img, shape, nf, res, k) in CASES_2D.items():
        img_out = os.path.join(HERE, "2d_" + os.path.basename(img) + ".gz")
        if not os.path.exists(img_out):
            with open(os.path.join(src, img), "rb") as fi, gzip.open(img_out, "wb", compresslevel=9) as fo:
                shutil.copyfileobj(fi, fo)
        nf_out = name + ".nf"
        shutil.copyfile(os.path.join(src, nf), os.path.join(HERE, nf_out))
        vals = np.fromfile(os.path.join(src, res), dtype=np.float64)
        manifest[name] = {
            "image": os.path.basename(img_out),
            "shape_yx": list(shape),
            "nf": nf_out,
            "tensor": [[float(v) for v in row] for row in vals[: k * k].reshape(k, k)],
            "reference_tolerance": 1e-4,
            "source": f"test/input/{res}",
        }
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CHFEM_REFERENCE", "/root/reference"))
