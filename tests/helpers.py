"""Test helpers: golden fixtures, the oracle (CPU checker) and small synthetic cases.

The oracle is only ever used here as the checker: the reference's own host code plus the CPU
restatement of its solver (oracle/_ref/chfem_oracle_exec, liboracle_ref.so), run in child
processes so its symbols never meet the product libraries.
"""
import ctypes
import gzip
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_EXEC = os.path.join(ROOT, "oracle", "_ref", "chfem_oracle_exec")
ORACLE_REF_LIB = os.path.join(ROOT, "oracle", "_ref", "liboracle_ref.so")
DROPIN_EXEC = os.path.join(ROOT, "oracle", "_ref", "chfem_exec_dropin")
CHFEM_EXEC = os.path.join(ROOT, "chfem_b200", "lib", "chfem_exec")


def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def golden_case_files(name, workdir):
    """Materialise a golden case (.nf + .raw) in workdir; returns (nf, raw, meta)."""
    meta = golden()[name]
    raw = os.path.join(workdir, meta["image"][:-3])
    if not os.path.exists(raw):
        with gzip.open(os.path.join(GOLDEN, meta["image"])) as f, open(raw, "wb") as g:
            shutil.copyfileobj(f, g)
    nf = os.path.join(workdir, meta["nf"])
    shutil.copy(os.path.join(GOLDEN, meta["nf"]), nf)
    return nf, raw, meta


def rel_to_max(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def run_exec(exe, nf, raw, *args, env=None, timeout=1800):
    """Run a chfem_exec-style CLI and return (C matrix, stdout)."""
    out = tempfile.mktemp(suffix=".bin")
    e = dict(os.environ)
    if env:
        e.update(env)
    p = subprocess.run([exe, nf, raw, "-b", out, *[str(a) for a in args]], capture_output=True, text=True,
                       timeout=timeout, env=e)
    if p.returncode != 0 or not os.path.exists(out):
        raise RuntimeError(f"{exe} failed ({p.returncode}):\n{p.stdout[-3000:]}\n{p.stderr[-3000:]}")
    C = np.fromfile(out)
    os.remove(out)
    k = int(round(np.sqrt(C.size)))
    return C[: k * k].reshape(k, k), p.stdout


def oracle_available():
    return os.path.exists(ORACLE_EXEC) and os.path.exists(ORACLE_REF_LIB)


# ---- oracle captures, computed in a child process -------------------------------------
_CAPTURE_SCRIPT = r'''
import ctypes, sys, json, numpy as np
lib = ctypes.CDLL(sys.argv[1], mode=ctypes.RTLD_LOCAL)
nf, raw, direction, out = sys.argv[2], sys.argv[3], int(sys.argv[4]), sys.argv[5]
lib.hmgInit.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p]
lib.oracle_set_quiet(1)
assert lib.hmgInit(nf.encode(), raw.encode(), None, None)
lib.hmgSetHomogenizationFlag(direction)
lib.hmgSolveHomogenization()
res = {}
sizes = {0: 2, 1: 4, 2: 4, 3: 1, 4: 8, 5: 8, 6: 8}
dt = {0: np.uint16, 1: np.uint32, 2: np.uint32, 3: np.uint8, 4: np.float64, 5: np.float64, 6: np.float64}
arrs = {}
for w in range(7):
    n = lib.oracle_captured_count(w)
    a = np.zeros(n, dtype=dt[w])
    if n:
        lib.oracle_copy_captured(w, a.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(n * sizes[w]))
    arrs[str(w)] = a
lib.hmgGetConstitutiveMtx.restype = ctypes.POINTER(ctypes.c_double)
lib.hmgGetConstitutiveMtxDim.restype = ctypes.c_uint
d = lib.hmgGetConstitutiveMtxDim()
C = np.ctypeslib.as_array(lib.hmgGetConstitutiveMtx(), shape=(d,)).copy()
arrs["C"] = C
lib.hmgGetThermalExpansion.restype = ctypes.POINTER(ctypes.c_double)
lib.hmgGetThermalExpansionDim.restype = ctypes.c_uint
na = lib.hmgGetThermalExpansionDim()
if na:
    arrs["alpha"] = np.ctypeslib.as_array(lib.hmgGetThermalExpansion(), shape=(na,)).copy()
np.savez(out, **arrs)
'''


def oracle_capture(nf, raw, direction):
    """Run the reference host code + CPU oracle solver on one load case; returns the arrays the
    host code handed over the cudapcg ABI (keys, maps, local matrices, RHS, solution) and C."""
    out = tempfile.mktemp(suffix=".npz")
    p = subprocess.run([sys.executable, "-c", _CAPTURE_SCRIPT, ORACLE_REF_LIB, nf, raw, str(direction), out],
                       capture_output=True, text=True, timeout=1800, env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
    if p.returncode != 0:
        raise RuntimeError(p.stdout[-2000:] + p.stderr[-2000:])
    z = np.load(out)
    res = {k: z[k] for k in z.files}
    os.remove(out)
    return res


# ---- small synthetic cases -------------------------------------------------------------
def small_image(shape, nmat, seed, codes=None):
    rng = np.random.default_rng(seed)
    codes = codes or [0, 255, 100, 50][:nmat]
    lab = rng.integers(0, nmat, size=shape)
    return np.array(codes, dtype=np.uint8)[lab]


def write_small_case(workdir, name, img, analysis, tol=1e-8, maxit=20000, solver=0, refinement=1, voxel=1.0, props=None):
    from chfem_b200.io import export_for_chfem
    codes = sorted(np.unique(img).tolist())
    if props is None:
        if analysis == 0:
            props = {c: [1.0, 10.0, 3.0, 0.5][i] for i, c in enumerate(codes)}
        elif analysis == 1:
            props = {c: [(1.0, 0.3), (10.0, 0.2), (4.0, 0.25), (0.5, 0.35)][i] for i, c in enumerate(codes)}
        else:
            props = None
    prefix = os.path.join(workdir, name)
    export_for_chfem(prefix + ".raw", img, analysis, mat_props=props, voxel_size=voxel, solver_type=solver,
                     refinement=refinement, export_raw=True, export_nf=True, solver_tolerance=tol,
                     solver_maxiter=maxit)
    return prefix + ".nf", prefix + ".raw"


def parse_iterations(log):
    """Iteration counts printed by a solve ("iteration: N, residual: ...")."""
    import re
    return [int(m) for m in re.findall(r"iteration: (\d+), residual", log)]
