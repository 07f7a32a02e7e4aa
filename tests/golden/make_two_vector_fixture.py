"""Generate tests/golden/two_vector_ref.json: the reference's own CUDA build run with the
2-vector Stokes solvers (CG2 / MINRES2, every x-reduce mode, with and without Jacobi, the three
stopping norms, an imported initial guess) on two small seeded pore images; with --2d,
tests/golden/two_vector_2d_ref.json from two seeded 2D pore images (pixels).

Needs a GPU and oracle/_ref/chfem_exec_ref (make -C oracle refgpu):

    python tests/golden/make_two_vector_fixture.py [--2d] [out.json]

For each run the fixture keeps the effective permeability tensor, the per-load-case iteration
counts and, for some runs, the per-step reductions the reference writes to
<nf>_xreduce_metrics_<n>.bin.  The tests pin the CPU oracle's restatement of these solvers on
it and then check the B200 library against the oracle.
"""
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

REF_EXEC = os.path.join(ROOT, "oracle", "_ref", "chfem_exec_ref")
CASES = {
    "pore16": dict(shape=(16, 18, 20), corr=2.0, porosity=0.45, seed=7, voxel=1.0, tol=1e-8),
    "pore12_h05": dict(shape=(12, 14, 10), corr=2.0, porosity=0.5, seed=21, voxel=0.5, tol=1e-9),
}
FLAGS = [
    ["-s", "1"], ["-s", "0"],
    ["-s", "5"], ["-s", "5", "-u", "0"], ["-s", "5", "-u", "1"], ["-s", "5", "-j", "0"], ["-s", "5", "-c", "1"],
    ["-s", "5", "-c", "2"],
    ["-s", "4"], ["-s", "4", "-u", "0"], ["-s", "4", "-u", "1"], ["-s", "4", "-j", "0"], ["-s", "4", "-c", "1"],
    ["-s", "4", "-c", "2"],
]
CASES_2D = {
    "pix30x26": dict(shape=(30, 26), porosity=0.6, seed=5, voxel=1.0, tol=1e-8),
    "pix22x35_h05": dict(shape=(22, 35), porosity=0.65, seed=17, voxel=0.5, tol=1e-9),
}
KEEP_METRICS = [["-s", "5"], ["-s", "5", "-u", "0"], ["-s", "4", "-u", "1"]]


def image(spec):
    """3D: a percolating Gaussian-random-field pore space; 2D: seeded uniform pixels."""
    if len(spec["shape"]) == 2:
        rng = np.random.default_rng(spec["seed"])
        return np.where(rng.random(spec["shape"]) < spec["porosity"], 0, 255).astype(np.uint8)
    from chfem_b200.synthetic import pore_grf
    return pore_grf(spec["shape"], corr=spec["corr"], porosity=spec["porosity"], seed=spec["seed"])


def make_case(workdir, name, spec):
    from chfem_b200.io import export_for_chfem
    img = image(spec)
    prefix = os.path.join(workdir, name)
    export_for_chfem(prefix + ".raw", img, 2, mat_props=None, voxel_size=spec["voxel"], solver_type=1, refinement=1,
                     export_raw=True, export_nf=True, solver_tolerance=spec["tol"], solver_maxiter=20000)
    return prefix + ".nf", prefix + ".raw"


def guess_settings(workdir, name, spec):
    """Same model, 20 iterations at most: the .nf file of the initial-guess run."""
    from chfem_b200.io import export_for_chfem
    img = image(spec)
    prefix = os.path.join(workdir, name + "_guess")
    export_for_chfem(prefix + ".raw", img, 2, mat_props=None, voxel_size=spec["voxel"], solver_type=1, refinement=1,
                     export_raw=False, export_nf=True, solver_tolerance=spec["tol"], solver_maxiter=20)
    return prefix + ".nf"


def run(nf, raw, flags):
    out = tempfile.mktemp(suffix=".bin")
    p = subprocess.run([REF_EXEC, nf, raw, "-b", out, *flags], capture_output=True, text=True, timeout=600)
    if p.returncode != 0 or not os.path.exists(out):
        raise RuntimeError(p.stdout[-2000:] + p.stderr[-2000:])
    v = np.fromfile(out)
    k = 2 if v.size == 4 else 3
    C = v[:k * k].reshape(k, k)
    os.remove(out)
    its = [int(m) for m in re.findall(r"iteration: (\d+), residual", p.stdout)]
    return C, its


def main():
    args = [a for a in sys.argv[1:] if a != "--2d"]
    dim2 = "--2d" in sys.argv[1:]
    default = "two_vector_2d_ref.json" if dim2 else "two_vector_ref.json"
    out_path = args[0] if args else os.path.join(ROOT, "tests", "golden", default)
    work = tempfile.mkdtemp()
    fixture = {"generator": "tests/golden/make_two_vector_fixture.py" + (" --2d" if dim2 else ""), "cases": {}}
    for name, spec in (CASES_2D if dim2 else CASES).items():
        nf, raw = make_case(work, name, spec)
        runs = []
        for flags in FLAGS:
            for f in os.listdir(work):
                if "_xreduce_metrics_" in f:
                    os.remove(os.path.join(work, f))
            C, its = run(nf, raw, flags)
            entry = {"flags": flags, "C": C.tolist(), "iterations": its}
            if flags in KEEP_METRICS:
                ncase = C.shape[0]  # load cases of the run: one metrics file each
                entry["metrics"] = [np.fromfile(os.path.join(work, f"{name}_xreduce_metrics_{k}.bin")).tolist()
                                    for k in range(1, ncase + 1)]
            runs.append(entry)
            print(name, flags, its, np.diag(C).tolist(), flush=True)
        # an imported initial guess: 20 MINRES steps (-xo, a settings file capped at 20
        # iterations), read back by MINRES2 / CG2 (-xi)
        nf20 = guess_settings(work, name, spec)
        run(nf20, raw, ["-s", "1", "-xo"])
        for flags in (["-s", "5"], ["-s", "4"]):
            C, its = run(nf, raw, [*flags, "-xi", nf20[:-3] + "_X"])
            runs.append({"flags": [*flags, "-xi", "<guess>_X"], "C": C.tolist(), "iterations": its})
        fixture["cases"][name] = {"spec": spec, "runs": runs}
    with open(out_path, "w") as f:
        json.dump(fixture, f, indent=0)
    shutil.rmtree(work)
    print("wrote", out_path)


if __name__ == "__main__":
    main()
