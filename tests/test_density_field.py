"""Scalar density field (-f; chfem's femhmg.c:1760-1835).

CPU: the 16-bit density codes and their range built by this library's host layer equal, bit
for bit, those the reference's own host code hands to the solver (captured by the oracle) --
refinement 1 and 2, float32 and float64 files, thermal and elastic.

GPU (marked gpu): the solutions of every load case (-xo) equal the oracle's (the reference's
host code and right-hand sides with the CPU restatement of its density-field operator,
matrix_free.cu:2270-2390 and :3091-3430) at 1e-6 relative to their largest entry; a field of
ones reproduces the two-phase model's tensor (each voxel's product is then its own phase
property, quantised exactly at the two ends of the range); the tensors of the columns the
reference computes consistently equal the oracle's at 1e-6.  The reference's tensor update
under a density field has defects (thermal: the flux coefficient of every voxel is read at
one stale voxel index, femhmg_thermal_3D.c:574,583; elastic, load case X: two terms miss the
density factor, femhmg_elastic_3D.c:1389); this library scales every voxel's terms by
its own density, so those columns are checked by the field-of-ones identity only.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from tests import helpers as H

_CAPTURE = r'''
import ctypes, sys, numpy as np
lib = ctypes.CDLL(sys.argv[1], mode=ctypes.RTLD_LOCAL)
lib.hmgInit.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p]
lib.oracle_set_quiet(1)
assert lib.hmgInit(sys.argv[2].encode(), sys.argv[3].encode(), sys.argv[4].encode(), None)
lib.hmgSetHomogenizationFlag(0)
lib.hmgSolveHomogenization()
n = lib.oracle_captured_count(7)
q = np.zeros(n, np.uint16)
lib.oracle_copy_captured(7, q.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(2 * n))
rg = np.zeros(2)
lib.oracle_copy_captured(8, rg.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(16))
np.savez(sys.argv[5], q=q, rg=rg)
'''


def make_case(tmp_path, analysis, shape, refinement, dtype, seed=5, field=None):
    from chfem_b200.io import export_for_chfem
    rng = np.random.default_rng(seed)
    img = np.where(rng.random(shape) < 0.4, 255, 0).astype(np.uint8)
    props = {0: 1.0, 255: 10.0} if analysis == 0 else {0: (1.0, 0.3), 255: (10.0, 0.2)}
    prefix = str(tmp_path / f"d{analysis}{refinement}{dtype}")
    export_for_chfem(prefix + ".raw", img, analysis, mat_props=props, voxel_size=1.0, refinement=refinement,
                     solver_tolerance=1e-10, solver_maxiter=20000)
    with open(prefix + ".nf", "a") as f:
        f.write(f"\n%data_type {dtype}\n")
    n = img.size * refinement ** img.ndim  # the reference reads as many values as the refined model has voxels
    vals = field if field is not None else 0.5 + rng.random(n)
    vals = np.resize(np.asarray(vals, float), n)
    vals.astype(np.float32 if dtype == "float32" else np.float64).tofile(prefix + ".bin")
    return prefix + ".nf", prefix + ".raw", prefix + ".bin"


@pytest.mark.skipif(not H.oracle_available(), reason="oracle not built")
@pytest.mark.parametrize("analysis,refinement,dtype,shape", [(0, 1, "float32", (5, 6, 7)), (1, 1, "float64", (5, 6, 7)),
                                                             (0, 2, "float64", (5, 6, 7)), (1, 2, "float32", (5, 6, 7)),
                                                             (0, 1, "float64", (9, 11)), (1, 2, "float32", (7, 6)),
                                                             (0, 3, "float32", (4, 5))])
def test_density_codes_equal_reference(tmp_path, analysis, refinement, dtype, shape):
    from chfem_b200 import _native
    nf, raw, fb = make_case(tmp_path, analysis, shape, refinement, dtype)
    out = str(tmp_path / "cap.npz")
    p = subprocess.run([sys.executable, "-c", _CAPTURE, H.ORACLE_REF_LIB, nf, raw, fb, out], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    ref = np.load(out)
    lib = _native.chfem()
    lib.chfemB200SetQuiet(1)
    lib.hmgInit.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p]
    assert lib.hmgInit(nf.encode(), raw.encode(), fb.encode(), None), lib.chfemB200LastError()
    n = lib.chfemB200ModelArraySize(8) // 2
    q = np.zeros(n, np.uint16)
    lib.chfemB200CopyModelArray(8, q.ctypes.data_as(ctypes.c_void_p), 2 * n)
    rg = np.zeros(2)
    lib.chfemB200CopyModelArray(9, rg.ctypes.data_as(ctypes.c_void_p), 16)
    lib.hmgEnd()
    assert np.array_equal(q, ref["q"])
    assert np.array_equal(rg, ref["rg"])


def _x_of(exe, nf, raw, fb, extra=(), dim=3):
    C, log = H.run_exec(exe, nf, raw, "-f", fb, "-xo", *extra)
    if dim == 2:  # 2D load cases: thermal X, Y; elastic X, Y, XY (files _0, _1, _5)
        dirs = [0, 1] if C.shape[0] == 2 else [0, 1, 5]
    else:
        dirs = list(range(C.shape[0] if C.shape[0] == 3 else 6))
    base = nf[:-3] + "_X"
    xs = [np.fromfile(f"{base}_{d}.bin") for d in dirs]
    for d in dirs:
        os.remove(f"{base}_{d}.bin")
    return C, xs, log


@pytest.mark.gpu
@pytest.mark.parametrize("analysis,refinement,extra", [(0, 1, []), (1, 1, []), (0, 2, []), (1, 1, ["-s", "2"]), (0, 1, ["-j", "0"])])
def test_density_solutions_equal_oracle(tmp_path, analysis, refinement, extra):
    nf, raw, fb = make_case(tmp_path, analysis, (7, 8, 9), refinement, "float32")
    # same solver flags on both sides: the periodic thermal solution is defined up to a constant,
    # which CG and PCG settle differently
    Cref, xref, logref = _x_of(H.ORACLE_EXEC, nf, raw, fb, extra)
    C, xs, log = _x_of(H.CHFEM_EXEC, nf, raw, fb, extra)
    for a, b in zip(xs, xref):
        assert H.rel_to_max(a, b) < 1e-6
    if analysis == 1:  # the columns the reference updates with each voxel's own density
        assert H.rel_to_max(C[:, 1:], Cref[:, 1:]) < 1e-6
    its, its_ref = H.parse_iterations(log), H.parse_iterations(logref)
    assert all(abs(a - b) <= 1 for a, b in zip(its, its_ref)), (its, its_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("analysis", [0, 1])
def test_density_of_ones_is_the_two_phase_model(tmp_path, analysis):
    nf, raw, fb = make_case(tmp_path, analysis, (7, 8, 9), 1, "float32", field=np.ones(1))
    Cplain, _ = H.run_exec(H.CHFEM_EXEC, nf, raw)
    Cf, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-f", fb)
    assert H.rel_to_max(Cf, Cplain) < 1e-6
    Cf_mixed, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-f", fb, "--precision", "mixed")
    assert H.rel_to_max(Cf_mixed, Cplain) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("analysis", [0, 1])
def test_density_field_minres(tmp_path, analysis):
    """MINRES under a density field: the solutions of every load case equal the oracle's
    (unpreconditioned: the reference's thermal / elastic PMINRES iterates with a stub inverse
    Jacobi, wrappers.cu:635-648); PMINRES gives the PCG solution."""
    nf, raw, fb = make_case(tmp_path, analysis, (6, 7, 8), 1, "float32")
    Cref, xref, logref = _x_of(H.ORACLE_EXEC, nf, raw, fb, ["-s", "1", "-j", "0"])
    C, xs, log = _x_of(H.CHFEM_EXEC, nf, raw, fb, ["-s", "1", "-j", "0"])
    for a, b in zip(xs, xref):
        assert H.rel_to_max(a, b) < 1e-6
    its, its_ref = H.parse_iterations(log), H.parse_iterations(logref)
    assert all(abs(a - b) <= max(1, 0.01 * b) for a, b in zip(its, its_ref)), (its, its_ref)
    Cp, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-f", fb)
    Cm, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-f", fb, "-s", "1")
    assert H.rel_to_max(Cm, Cp) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("analysis,refinement,extra", [(0, 1, []), (1, 1, []), (0, 2, []), (1, 1, ["-s", "2"]),
                                                       (1, 1, ["-j", "0"]), (1, 1, ["--precision", "mixed"])])
def test_density_2d_equal_oracle(tmp_path, analysis, refinement, extra):
    """2D images (femhmg_thermal_2D.c / femhmg_elastic_2D.c *_ScalarDensityField,
    matrix_free.cu:1800-1880, :2748-2850): solutions of every load case and the whole tensor
    (the reference's 2D updates scale each pixel by its own density) against the oracle."""
    nf, raw, fb = make_case(tmp_path, analysis, (23, 19), refinement, "float32")
    flags = [f for f in extra if f not in ("--precision", "mixed")]
    Cref, xref, logref = _x_of(H.ORACLE_EXEC, nf, raw, fb, flags, dim=2)
    C, xs, log = _x_of(H.CHFEM_EXEC, nf, raw, fb, extra, dim=2)
    tol = 1e-4 if "mixed" in extra else 1e-6
    for a, b in zip(xs, xref):
        assert H.rel_to_max(a, b) < tol
    assert H.rel_to_max(C, Cref) < tol
    if "mixed" not in extra:
        its, its_ref = H.parse_iterations(log), H.parse_iterations(logref)
        assert all(abs(a - b) <= 1 for a, b in zip(its, its_ref)), (its, its_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("analysis", [0, 1])
def test_density_2d_minres_and_ones(tmp_path, analysis):
    """2D: MINRES without Jacobi equals the oracle's; a field of ones gives the two-phase
    tensor; PMINRES gives the PCG tensor."""
    nf, raw, fb = make_case(tmp_path, analysis, (17, 21), 1, "float32")
    Cref, xref, _ = _x_of(H.ORACLE_EXEC, nf, raw, fb, ["-s", "1", "-j", "0"], dim=2)
    C, xs, _ = _x_of(H.CHFEM_EXEC, nf, raw, fb, ["-s", "1", "-j", "0"], dim=2)
    for a, b in zip(xs, xref):
        assert H.rel_to_max(a, b) < 1e-6
    Cp, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-f", fb)
    Cm, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-f", fb, "-s", "1")
    assert H.rel_to_max(Cm, Cp) < 1e-6
    nf1, raw1, fb1 = make_case(tmp_path, analysis, (17, 21), 1, "float32", field=np.ones(1))
    Cplain, _ = H.run_exec(H.CHFEM_EXEC, nf1, raw1)
    Cf, _ = H.run_exec(H.CHFEM_EXEC, nf1, raw1, "-f", fb1)
    assert H.rel_to_max(Cf, Cplain) < 1e-6


@pytest.mark.gpu
def test_density_field_warnings_as_reference(tmp_path):
    """-e and -r with a density field print the reference's warnings and carry on (no field
    files, zero guess), with the tensor of the plain run."""
    import glob
    nf, raw, fb = make_case(tmp_path, 0, (6, 7, 8), 1, "float32")
    C, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-f", fb)
    Ce, loge = H.run_exec(H.CHFEM_EXEC, nf, raw, "-f", fb, "-e")
    assert "Field exportation not supported for scalar field input" in loge
    assert not glob.glob(str(tmp_path / "*_flux_*.bin"))
    Cr, logr = H.run_exec(H.CHFEM_EXEC, nf, raw, "-f", fb, "-r", "1")
    assert "Initial guess estimation is not yet available for analyses with a scalar field input" in logr
    assert H.rel_to_max(Ce, C) < 1e-12 and H.rel_to_max(Cr, C) < 1e-12
