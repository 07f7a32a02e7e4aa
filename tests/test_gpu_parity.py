"""GPU parity of chfem_b200 against the oracle (GPU box; marked gpu).

Bars (stated per test): FP64 effective tensors within 1e-6 relative to the largest entry of
the oracle's tensor, mixed precision within 1e-4; operator applies within 1e-12 (FP64) and
1e-5 (FP32 storage) relative to the largest entry; maps and DOF counts bit-exact (checked on
the CPU in test_host_parity.py).  The oracle is the reference's host code plus the CPU
restatement of its solver, run as a child process.
"""
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import zlib

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-6
MIXED_TOL = 1e-4


def oracle_columns():
    with open(os.path.join(H.GOLDEN, "oracle_columns.json")) as f:
        return json.load(f)


# ---------------------------------------------------------------------------------------
# Golden cases through the product CLI (chfem_b200/lib/chfem_exec)
@pytest.mark.parametrize("key,precision", [
    ("thermal_x_pcg", "fp64"), ("elastic_y_pcg", "fp64"), ("fluid_z_pcg", "fp64"), ("fluid_z_pminres", "fp64"),
    ("thermal_all_pcg", "fp64"), ("thermal_x_pcg", "mixed"), ("elastic_y_pcg", "mixed"), ("fluid_z_pminres", "mixed"),
])
def test_golden_cases(tmp_path, key, precision):
    ref = oracle_columns()[key]
    nf, raw, meta = H.golden_case_files(ref["case"], str(tmp_path))
    C, log = H.run_exec(H.CHFEM_EXEC, nf, raw, *ref["flags"], "--precision", precision)
    Cref = np.array(ref["C"])
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    cols = [meta["direction"]] if "-d" in ref["flags"] else list(range(Cref.shape[1]))
    solve_tol = nf_tolerance(nf)
    for c in cols:
        if precision == "mixed" and solve_tol > 1e-5:
            # A solve stopped at relative residual tol fixes the tensor to O(tol): the loaded
            # (largest) entry still meets the mixed bar, the near-zero entries of the column
            # agree to 10 tol between two valid iteration paths (FP64 and mixed).
            i = int(np.argmax(np.abs(Cref[:, c])))
            assert abs(C[i, c] - Cref[i, c]) / abs(Cref[i, c]) < MIXED_TOL, (c, C[:, c], Cref[:, c])
            assert H.rel_to_max(C[:, c], Cref[:, c]) < 10 * solve_tol, (c, C[:, c], Cref[:, c])
        else:
            assert H.rel_to_max(C[:, c], Cref[:, c]) < tol, (c, C[:, c], Cref[:, c])
    # and within the reference's own regression bar of its golden column (for mixed precision
    # at a loose solve tolerance, with the same split as above)
    gcol = np.array(meta["column"])
    cd = C[:, meta["direction"]]
    if precision == "mixed" and solve_tol > 1e-5:
        i = int(np.argmax(np.abs(gcol)))
        assert abs(cd[i] - gcol[i]) / abs(gcol[i]) < meta["reference_tolerance"]
        assert H.rel_to_max(cd, gcol) < 10 * solve_tol
    else:
        assert H.rel_to_max(cd, gcol) < meta["reference_tolerance"]
    if precision == "fp64":  # same recurrence, same stopping test: same iteration counts (+-1 for round-off)
        its = H.parse_iterations(log)
        assert len(its) == len(ref["iterations"])
        assert all(abs(a - b) <= 1 for a, b in zip(its, ref["iterations"])), (its, ref["iterations"])


def nf_tolerance(nf):
    lines = open(nf).read().split()
    return float(lines[lines.index("%solver_tolerance") + 1])


def test_python_api_golden(tmp_path):
    """compute_property with nf_filepath, like the reference's test/test_chfem.py:6-10."""
    from chfem_b200 import compute_property, import_raw
    ref = oracle_columns()["thermal_x_pcg"]
    nf, raw, meta = H.golden_case_files("thermal_ggg40", str(tmp_path))
    arr = import_raw(raw, (100, 100, 100))
    C = np.array(compute_property("conductivity", arr, direction="x", nf_filepath=nf))
    assert H.rel_to_max(C[:, 0], np.array(ref["C"])[:, 0]) < FP64_TOL


# ---------------------------------------------------------------------------------------
# Small synthetic models: every analysis x solver x option, product CLI versus oracle CLI
SMALL = [
    # name, analysis, builder, cli flags
    ("th2_pcg", 0, ("img", (14, 17, 19), 2), ["-d", "6"]),
    ("th4_cg", 0, ("img", (9, 13, 7), 4), ["-j", "0"]),
    ("th3_minres", 0, ("img", (10, 11, 12), 3), ["-s", "1", "-j", "0"]),
    ("th2_inf", 0, ("img", (12, 12, 12), 2), ["-c", "1"]),
    ("th2_err", 0, ("img", (12, 10, 9), 2), ["-c", "2"]),
    ("th2_ebe", 0, ("img", (11, 9, 13), 2), ["-p", "1"]),
    ("th_thin", 0, ("img", (1, 2, 33), 2), []),
    ("el2_pcg", 1, ("img", (10, 12, 11), 2), []),
    ("el4_pcg", 1, ("img", (7, 9, 8), 4), ["-d", "3"]),
    ("el2_ebe", 1, ("img", (8, 8, 9), 2), ["-p", "1", "-d", "5"]),
    ("fl_pcg", 2, ("pore", (16, 18, 20), 0.45), ["-s", "0"]),
    ("fl_pminres", 2, ("pore", (16, 18, 20), 0.45), ["-s", "1"]),
    ("fl_minres_nopre", 2, ("pore", (14, 14, 14), 0.5), ["-s", "1", "-j", "0", "-d", "0"]),
]


def build_small(tmp_path, name, analysis, spec):
    if spec[0] == "img":
        img = H.small_image(spec[1], spec[2], seed=zlib.crc32(name.encode()) % 10000)
    else:
        from chfem_b200.synthetic import pore_grf
        img = pore_grf(spec[1], corr=2.0, porosity=spec[2], seed=zlib.crc32(name.encode()) % 10000)
    return H.write_small_case(str(tmp_path), name, img, analysis, tol=1e-8, maxit=20000)


@pytest.mark.parametrize("name,analysis,spec,flags", SMALL)
def test_small_models_fp64(tmp_path, name, analysis, spec, flags):
    nf, raw = build_small(tmp_path, name, analysis, spec)
    Cref, _ = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags)
    C, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, *flags)
    assert H.rel_to_max(C, Cref) < FP64_TOL


@pytest.mark.parametrize("name,analysis,spec,flags", [s for s in SMALL if s[0] in ("th2_pcg", "el2_pcg", "fl_pminres")])
def test_small_models_mixed(tmp_path, name, analysis, spec, flags):
    nf, raw = build_small(tmp_path, name, analysis, spec)
    Cref, logref = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags)
    C, log = H.run_exec(H.CHFEM_EXEC, nf, raw, *flags, "--precision", "mixed")
    assert H.rel_to_max(C, Cref) < MIXED_TOL
    assert_mixed_converges(log, logref)


def assert_mixed_converges(log, logref):
    """Mixed precision reaches the tolerance (no stall up to the iteration cap) in at most
    twice the FP64 iteration count plus one restart cycle."""
    its, its_ref = H.parse_iterations(log), H.parse_iterations(logref)
    assert len(its) == len(its_ref)
    assert all(a <= 2 * b + 50 for a, b in zip(its, its_ref)), (its, its_ref)


def test_homogeneous_is_exact(tmp_path):
    """A one-phase image has the phase's own tensor: k I for conduction."""
    img = np.zeros((8, 9, 10), np.uint8)
    from chfem_b200.io import export_for_chfem
    export_for_chfem(str(tmp_path / "h.raw"), img, 0, mat_props={0: 3.5}, solver_tolerance=1e-10, solver_maxiter=1000)
    C, log = H.run_exec(H.CHFEM_EXEC, str(tmp_path / "h.nf"), str(tmp_path / "h.raw"))
    assert np.allclose(C, 3.5 * np.eye(3), atol=1e-9)


def test_initial_guess_roundtrip(tmp_path):
    """-xo writes x per load case; -xi reads it back and the solve stops at once with the same tensor."""
    nf, raw = build_small(tmp_path, "x0", 1, ("img", (8, 9, 10), 2))
    C1, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-d", "2", "-xo")
    prefix = nf[:-3] + "_X"
    assert os.path.exists(prefix + "_2.bin")
    C2, log = H.run_exec(H.CHFEM_EXEC, nf, raw, "-d", "2", "-xi", prefix)
    assert "Initial guess satisfied" in log
    assert H.rel_to_max(C2[:, 2], C1[:, 2]) < 1e-12


def test_dropin_reference_host_on_b200_library(tmp_path):
    """The reference's unmodified host code + CLI (femhmg + main.c) linked against
    libcudapcg_b200.so reproduces the oracle."""
    if not os.path.exists(H.DROPIN_EXEC):
        pytest.skip("drop-in executable not built (needs the reference tree at build time)")
    for name, analysis, spec, flags in [SMALL[0], SMALL[7], SMALL[11]]:
        nf, raw = build_small(tmp_path, name, analysis, spec)
        Cref, _ = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags)
        C, _ = H.run_exec(H.DROPIN_EXEC, nf, raw, *flags)
        assert H.rel_to_max(C, Cref) < FP64_TOL


# ---------------------------------------------------------------------------------------
# Operator and preconditioner applies through the C ABI, versus the standalone oracle
from chfem_b200._native import setup_cudapcg_model as setup_model  # noqa: E402


_ORACLE_APPLY = r'''
import ctypes, sys, pickle, numpy as np
sys.path.insert(0, sys.argv[3])
from tests.test_gpu_parity import setup_model
a = pickle.load(open(sys.argv[1], "rb"))
lib = ctypes.CDLL(sys.argv[2], mode=ctypes.RTLD_LOCAL)
setup_model(lib, a)
y = np.zeros(a["ndof"]); z = np.zeros(a["ndof"])
assert lib.oracle_apply(a["x"].ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p))
assert lib.oracle_precond(a["x"].ctypes.data_as(ctypes.c_void_p), z.ctypes.data_as(ctypes.c_void_p))
np.save(sys.argv[1] + ".y.npy", y); np.save(sys.argv[1] + ".z.npy", z)
'''


def host_arrays(nf, raw):
    from chfem_b200 import _native
    lib = _native.chfem()
    lib.chfemB200SetQuiet(1)
    assert lib.hmgInit(nf.encode(), raw.encode(), None, None)
    info = (ctypes.c_uint * 9)()
    lib.chfemB200ModelInfo(info)
    def arr(w, t):
        n = lib.chfemB200ModelArraySize(w)
        x = np.zeros(n // np.dtype(t).itemsize, dtype=t)
        if n:
            lib.chfemB200CopyModelArray(w, x.ctypes.data_as(ctypes.c_void_p), n)
        return x
    a = dict(nx=info[0], ny=info[1], nz=info[2], N=info[3], ndof=info[4], nV=info[5], nB=info[6], nkeys=max(1, info[7]) if info[8] != 2 else 1,
             analysis=info[8], keys=arr(0, np.uint16), dof_of_node=arr(1, np.uint32), node_of_dof=arr(2, np.uint32),
             border=arr(3, np.uint8), lcl=arr(4, np.float64))
    lib.hmgEnd()
    return a


@pytest.mark.parametrize("name,analysis,spec", [("th", 0, ("img", (13, 35, 17), 3)), ("el", 1, ("img", (9, 33, 10), 2)),
                                                 ("fl", 2, ("pore", (18, 20, 22), 0.45)), ("th_small", 0, ("img", (2, 3, 1), 2))])
@pytest.mark.parametrize("precision", [0, 1])
def test_operator_and_jacobi(tmp_path, name, analysis, spec, precision):
    import pickle
    from chfem_b200 import _native
    nf, raw = build_small(tmp_path, name, analysis, spec)
    a = host_arrays(nf, raw)
    rng = np.random.default_rng(5)
    a["x"] = rng.standard_normal(a["ndof"])
    pk = str(tmp_path / "a.pkl")
    pickle.dump(a, open(pk, "wb"))
    p = subprocess.run([sys.executable, "-c", _ORACLE_APPLY, pk, os.path.join(H.ROOT, "oracle", "liboracle_cudapcg.so"), H.ROOT],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    yref, zref = np.load(pk + ".y.npy"), np.load(pk + ".z.npy")
    lib = _native.cudapcg()
    setup_model(lib, a)
    assert lib.cudapcgB200SetPrecision(precision)
    y = np.zeros(a["ndof"]); z = np.zeros(a["ndof"])
    assert lib.cudapcgB200ApplyOperator(a["x"].ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p)), lib.cudapcgB200LastError()
    assert lib.cudapcgB200ApplyPreconditioner(a["x"].ctypes.data_as(ctypes.c_void_p), z.ctypes.data_as(ctypes.c_void_p))
    lib.cudapcgEnd()
    tol = 1e-12 if precision == 0 else 1e-5
    assert H.rel_to_max(y, yref) < tol
    assert H.rel_to_max(z, zref) < tol


@pytest.mark.parametrize("spec", [("img", (13, 35, 17), 4), ("img", (40, 9, 66), 2), ("img", (1, 2, 3), 3)])
@pytest.mark.parametrize("precision", [0, 1])
def test_thermal_pass_equals_generic(tmp_path, spec, precision, monkeypatch):
    """The thermal pass written for cubic-symmetric conduction matrices (stencil_th.cuh) against
    the oracle and against the generic thermal pass (CHFEM_B200_THERMAL_OP=generic), 2 to 4
    materials, thin and ragged shapes."""
    import pickle
    from chfem_b200 import _native
    nf, raw = build_small(tmp_path, "thp", 0, spec)
    a = host_arrays(nf, raw)
    a["x"] = np.random.default_rng(7).standard_normal(a["ndof"])
    pk = str(tmp_path / "a.pkl")
    pickle.dump(a, open(pk, "wb"))
    p = subprocess.run([sys.executable, "-c", _ORACLE_APPLY, pk, os.path.join(H.ROOT, "oracle", "liboracle_cudapcg.so"), H.ROOT],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    yref = np.load(pk + ".y.npy")
    lib = _native.cudapcg()
    ys = []
    for op in ("", "generic"):
        monkeypatch.setenv("CHFEM_B200_THERMAL_OP", op)
        setup_model(lib, a)
        assert lib.cudapcgB200SetPrecision(precision)
        y = np.zeros(a["ndof"])
        assert lib.cudapcgB200ApplyOperator(a["x"].ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p)), lib.cudapcgB200LastError()
        lib.cudapcgEnd()
        ys.append(y)
    tol = 1e-12 if precision == 0 else 1e-5
    assert H.rel_to_max(ys[0], yref) < tol
    assert H.rel_to_max(ys[1], yref) < tol
    assert H.rel_to_max(ys[0], ys[1]) < (1e-13 if precision == 0 else 1e-5)


_ORACLE_APPLY_MANY = r'''
import ctypes, sys, pickle, numpy as np
sys.path.insert(0, sys.argv[3])
from tests.test_gpu_parity import setup_model
a = pickle.load(open(sys.argv[1], "rb"))
lib = ctypes.CDLL(sys.argv[2], mode=ctypes.RTLD_LOCAL)
setup_model(lib, a)
ys = []
for x in a["xs"]:
    y = np.zeros(a["ndof"])
    assert lib.oracle_apply(np.ascontiguousarray(x).ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p))
    ys.append(y)
np.save(sys.argv[1] + ".ys.npy", np.array(ys))
'''


# The block operator pass of the block solver (for one- and two-material models the stencil
# assembled per material configuration, otherwise element by element), applied to 3 or 6
# random fields at once; each output against the oracle's single apply.  Bars as above.
@pytest.mark.parametrize("name,analysis,spec,nr", [
    ("th2", 0, ("img", (13, 35, 17), 2), 3), ("th1", 0, ("img", (9, 8, 11), 1), 3), ("th3", 0, ("img", (10, 33, 9), 3), 3),
    ("el2", 1, ("img", (9, 33, 10), 2), 6), ("el2_3", 1, ("img", (11, 7, 13), 2), 3), ("el4", 1, ("img", (7, 9, 8), 4), 6),
    ("el2_odd", 1, ("img", (33, 10, 7), 2), 6), ("th2_tiny", 0, ("img", (2, 3, 1), 2), 3)])
@pytest.mark.parametrize("precision", [0, 1])
def test_block_operator(tmp_path, name, analysis, spec, nr, precision):
    import pickle
    from chfem_b200 import _native
    nf, raw = build_small(tmp_path, name, analysis, spec)
    a = host_arrays(nf, raw)
    rng = np.random.default_rng(7)
    a["xs"] = [rng.standard_normal(a["ndof"]) for _ in range(nr)]
    pk = str(tmp_path / "a.pkl")
    pickle.dump(a, open(pk, "wb"))
    p = subprocess.run([sys.executable, "-c", _ORACLE_APPLY_MANY, pk, os.path.join(H.ROOT, "oracle", "liboracle_cudapcg.so"), H.ROOT],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    yref = np.load(pk + ".ys.npy")
    lib = _native.cudapcg()
    setup_model(lib, a)
    assert lib.cudapcgB200SetPrecision(precision)
    ys = [np.zeros(a["ndof"]) for _ in range(nr)]
    P = ctypes.c_void_p * nr
    ok = lib.cudapcgB200ApplyBlockOperator(nr, P(*[x.ctypes.data for x in a["xs"]]), P(*[y.ctypes.data for y in ys]))
    err = lib.cudapcgB200LastError()
    lib.cudapcgEnd()
    assert ok, err
    tol = 1e-12 if precision == 0 else 1e-5
    for k in range(nr):
        assert H.rel_to_max(ys[k], yref[k]) < tol, (k, H.rel_to_max(ys[k], yref[k]))


# ---------------------------------------------------------------------------------------
# Block multi-RHS solves (--multirhs): every load case advances in one pass, each with its
# own PCG scalars and stopping test.  Same bars as the one-by-one solves; FP64 iteration
# counts within +-1 of the oracle's (the FMA order of the block operator differs).
BLOCK = [s for s in SMALL if s[0] in ("th2_pcg", "th4_cg", "th2_inf", "th2_err", "th2_ebe", "th_thin", "el2_pcg")] + [
    ("el3_ebe_all", 1, ("img", (8, 8, 9), 3), ["-p", "1"]),
    ("el2_nopre", 1, ("img", (7, 6, 9), 2), ["-j", "0"]),
    ("fl_pminres", 2, ("pore", (16, 18, 20), 0.45), ["-s", "1"]),
    ("fl_minres_nopre_all", 2, ("pore", (14, 14, 14), 0.5), ["-s", "1", "-j", "0"]),
    ("fl_pminres_inf", 2, ("pore", (12, 16, 14), 0.5), ["-s", "1", "-c", "1"]),
]


@pytest.mark.parametrize("name,analysis,spec,flags", BLOCK)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_block_multirhs(tmp_path, name, analysis, spec, flags, precision):
    nf, raw = build_small(tmp_path, name, analysis, spec)
    Cref, logref = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags)
    C, log = H.run_exec(H.CHFEM_EXEC, nf, raw, *flags, "--multirhs", "--precision", precision)
    assert "Block solve" in log
    assert H.rel_to_max(C, Cref) < (FP64_TOL if precision == "fp64" else MIXED_TOL)
    if precision == "fp64":
        # +-1, or 3 % for the unpreconditioned Stokes MINRES cases, whose residual plateaus near
        # the tolerance make the stopping iteration sensitive to the summation order (of the
        # block operator here, of the oracle's OpenMP reductions there; observed 305 against 299)
        its, its_ref = H.parse_iterations(log), H.parse_iterations(logref)
        assert len(its) == len(its_ref)
        slack = 0.03 if "nopre" in name else 0.0
        assert all(abs(a - b) <= max(1, slack * b) for a, b in zip(its, its_ref)), (its, its_ref)
    else:
        assert_mixed_converges(log, logref)


@pytest.mark.parametrize("key", ["thermal_all_pcg"])
def test_block_multirhs_golden(tmp_path, key):
    ref = oracle_columns()[key]
    nf, raw, meta = H.golden_case_files(ref["case"], str(tmp_path))
    C, log = H.run_exec(H.CHFEM_EXEC, nf, raw, *ref["flags"], "--multirhs")
    assert "Block solve" in log
    assert H.rel_to_max(C, np.array(ref["C"])) < FP64_TOL


def test_block_multirhs_python_api():
    from chfem_b200 import compute_property
    img = H.small_image((10, 11, 12), 2, seed=3)
    C1 = np.array(compute_property("elasticity", img, mat_props={0: (10.0, 0.25), 255: (100.0, 0.3)}, solver_tolerance=1e-8))
    C2 = np.array(compute_property("elasticity", img, mat_props={0: (10.0, 0.25), 255: (100.0, 0.3)}, solver_tolerance=1e-8, multirhs=True))
    assert H.rel_to_max(C2, C1) < FP64_TOL


# ---------------------------------------------------------------------------------------
# Recursive coarse-grid initial guesses (-r N): the image coarsened by 2 per axis is solved
# first and its prolonged solution seeds the next finer level (femhmg.c:561-846).  Tensors to
# the FP64 bar and every level's iteration count within +-1 of the oracle's.
RECURSIVE = [
    ("th_r1", 0, ("img", (16, 18, 20), 2), ["-r", "1"]),
    ("th_r2_odd", 0, ("img", (17, 21, 19), 3), ["-r", "2"]),
    ("el_r1", 1, ("img", (12, 14, 10), 2), ["-r", "1"]),
    ("el_r1_dir", 1, ("img", (12, 10, 14), 2), ["-r", "1", "-d", "4"]),
    ("th_r1_cg", 0, ("img", (16, 16, 16), 2), ["-r", "1", "-j", "0"]),
]


@pytest.mark.parametrize("name,analysis,spec,flags", RECURSIVE)
@pytest.mark.parametrize("extra", [[], ["--multirhs"]])
def test_recursive_initial_guess(tmp_path, name, analysis, spec, flags, extra):
    if extra and "-d" in flags:
        pytest.skip("a single load case has no block")
    nf, raw = build_small(tmp_path, name, analysis, spec)
    Cref, logref = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags)
    C, log = H.run_exec(H.CHFEM_EXEC, nf, raw, *flags, *extra)
    assert H.rel_to_max(C, Cref) < FP64_TOL
    its, its_ref = H.parse_iterations(log), H.parse_iterations(logref)
    assert len(its) == len(its_ref) and len(its) > 0
    assert all(abs(a - b) <= 1 for a, b in zip(its, its_ref)), (its, its_ref)
    # from a zero guess: the same tensor, and the fine level needs at least as many iterations
    i = flags.index("-r")
    plain = flags[:i] + flags[i + 2:]
    C0, log0 = H.run_exec(H.CHFEM_EXEC, nf, raw, *plain, *extra)
    assert H.rel_to_max(C0, C) < FP64_TOL
    its0 = H.parse_iterations(log0)
    assert sum(its[-len(its0):]) <= sum(its0) + 2 * len(its0), (its, its0)


def test_block_export_roundtrip(tmp_path):
    """--multirhs with -xo brings every load case's x back to the host; -xi then starts each
    case at its solution, which the block solve accepts at once with the same tensor."""
    nf, raw = build_small(tmp_path, "xb", 1, ("img", (8, 9, 10), 2))
    C1, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "--multirhs", "-xo")
    prefix = nf[:-3] + "_X"
    assert all(os.path.exists(f"{prefix}_{d}.bin") for d in range(6))
    C2, log = H.run_exec(H.CHFEM_EXEC, nf, raw, "--multirhs", "-xi", prefix)
    assert log.count("Initial guess satisfied") == 6
    assert H.rel_to_max(C2, C1) < 1e-12


# ---------------------------------------------------------------------------------------
# Node keys built on the device from the image's colours (the one-call and block paths) are
# the host's keys bit for bit: the operator applied with either is identical.
@pytest.mark.parametrize("name,analysis,shape,nmat,refinement", [("th4", 0, (5, 7, 6), 4, 1), ("el3_ref2", 1, (3, 4, 5), 3, 2)])
def test_device_keys_from_colors(tmp_path, name, analysis, shape, nmat, refinement):
    from chfem_b200 import _native
    from chfem_b200.io import import_nf
    img = H.small_image(shape, nmat, seed=zlib.crc32(name.encode()) % 10000)
    nf, raw = H.write_small_case(str(tmp_path), name, img, analysis, refinement=refinement)
    a = host_arrays(nf, raw)
    lut = (ctypes.c_int * 256)(*([-1] * 256))  # colour -> material index
    for i, p in enumerate(import_nf(nf)["properties_of_materials"]):
        lut[p[0]] = i
    x = np.random.default_rng(2).standard_normal(a["ndof"])
    lib = _native.cudapcg()
    colors = np.ascontiguousarray(img.reshape(-1))
    nz, ny, nx = img.shape
    ys = []
    for device_keys in (False, True):
        setup_model(lib, a)
        if device_keys:
            assert lib.cudapcgB200SetImageColors(colors.ctypes.data_as(ctypes.c_void_p), ny, nx, nz, refinement, lut), \
                lib.cudapcgB200LastError()
        y = np.zeros(a["ndof"])
        assert lib.cudapcgB200ApplyOperator(x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p))
        lib.cudapcgEnd()
        ys.append(y)
    np.testing.assert_array_equal(ys[0], ys[1])
    # a colour outside the list is an error, not a key
    setup_model(lib, a)
    lut[int(colors[0])] = -1
    assert not lib.cudapcgB200SetImageColors(colors.ctypes.data_as(ctypes.c_void_p), ny, nx, nz, refinement, lut)
    lib.cudapcgEnd()
