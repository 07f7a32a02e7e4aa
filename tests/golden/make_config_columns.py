"""Effective tensors of the benchmark workloads computed by the oracle, for the GPU tests of
those configurations (tests/test_gpu_configs.py), which run where the oracle's CPU solves of
these 0.3-6 M DOF models would take minutes.

The oracle is the reference's own host code driving the CPU restatement of its solver
(oracle/_ref/chfem_oracle_exec, built by `make -C oracle ref`), FP64 PCG / MINRES with the
Jacobi preconditioner, every load case, at the workload's tolerance.  The images come from the
seeded generators of chfem_b200.synthetic; each entry records the image's CRC-32 so a test
regenerating it can tell that it solves the same image.
  thermal64_spheres  64^3 non-overlapping balls (r 4-8) at 30 % phase 1, k 1 / 10, seed 1000
  elastic128_grf     128^3 periodic GRF, correlation 6, 40 % phase 1, E/nu 1/0.30 and 10/0.20, seed 2000
  stokes64_grf       64^3 pore GRF, correlation 8, porosity 0.35 (percolating clusters), seed 3000
                     (the 128^3 Stokes workload's generator at 64^3, where the CPU solve is short)
Usage: python tests/golden/make_config_columns.py [name ...]
"""
import json
import os
import sys
import tempfile
import time
import zlib

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from tests import helpers as H  # noqa: E402

CONFIGS = {
    "thermal64_spheres": dict(analysis=0, gen="spheres", shape=(64, 64, 64), vf=0.30, seed=1000,
                              props={0: 1.0, 255: 10.0}, tol=1e-6, solver=0),
    "elastic128_grf": dict(analysis=1, gen="grf", shape=(128, 128, 128), corr=6.0, fraction=0.40, seed=2000,
                           props={0: (1.0, 0.30), 255: (10.0, 0.20)}, tol=1e-6, solver=0),
    "stokes64_grf": dict(analysis=2, gen="pore", shape=(64, 64, 64), corr=8.0, porosity=0.35, seed=3000,
                         props=None, tol=1e-6, solver=1),
}


def make_image(c):
    from chfem_b200 import synthetic
    if c["gen"] == "spheres":
        return synthetic.spheres(c["shape"], vf=c["vf"], seed=c["seed"])
    if c["gen"] == "grf":
        return synthetic.grf(c["shape"], corr=c["corr"], fraction=c["fraction"], seed=c["seed"])
    return synthetic.pore_grf(c["shape"], corr=c["corr"], porosity=c["porosity"], seed=c["seed"])


def write_case(wd, name, c, img):
    from chfem_b200.io import export_for_chfem
    prefix = os.path.join(wd, name)
    export_for_chfem(prefix + ".raw", img, c["analysis"], mat_props=c["props"], voxel_size=1.0, solver_type=c["solver"],
                     solver_tolerance=c["tol"], solver_maxiter=100000)
    return prefix + ".nf", prefix + ".raw"


def main(names):
    path = os.path.join(H.GOLDEN, "config_columns.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    with tempfile.TemporaryDirectory() as wd:
        for name in names:
            c = CONFIGS[name]
            img = make_image(c)
            nf, raw = write_case(wd, name, c, img)
            t0 = time.time()
            C, log = H.run_exec(H.ORACLE_EXEC, nf, raw, env={"OMP_NUM_THREADS": str(os.cpu_count() or 4)}, timeout=7200)
            its = H.parse_iterations(log)
            out[name] = {"config": {k: (list(v) if isinstance(v, tuple) else v) for k, v in c.items() if k != "props"},
                         "props": {str(k): v for k, v in (c["props"] or {}).items()},
                         "image_crc32": zlib.crc32(img.tobytes()), "C": C.tolist(), "iterations": its}
            print(name, its, f"{time.time() - t0:.0f} s", flush=True)
            with open(path, "w") as f:
                json.dump(out, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CONFIGS))
