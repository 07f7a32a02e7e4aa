"""Device memory per unknown of the solvers, and the 3-vector PCG (-s 2) that keeps the least.

The reference's PCG keeps x, r, d, q and s (40 B per unknown in FP64) and its 3-vector PCG
x, r and d (chfem/src/femhmg/cudapcg/solvers/pcg3.cu:28-227; 24 B, README.md:244-256).  Here
PCG keeps x, b, r, q and the direction's two buffers (M^-1 r is formed inside the operator
pass, never stored): 48 B in FP64; the 3-vector PCG x, r and the two direction buffers
(32 B), applying the operator twice per iteration as the reference's does.  Its iterates are
CG's, so its tensors and iteration counts are checked against the oracle's CG (the same bars
as the other GPU tests: FP64 1e-6, mixed 1e-4 relative to the largest entry; iterations +-1).
"""
import ctypes
import zlib

import numpy as np
import pytest

from tests import helpers as H
from tests.test_gpu_parity import FP64_TOL, MIXED_TOL, assert_mixed_converges, build_small, host_arrays

pytestmark = pytest.mark.gpu

CASES = [("th2", 0, ("img", (14, 17, 19), 2), []), ("el2", 1, ("img", (10, 12, 11), 2), []),
         ("el4", 1, ("img", (7, 9, 8), 4), ["-d", "3"]), ("th2_cg", 0, ("img", (12, 13, 10), 2), ["-j", "0"]),
         ("el2_inf", 1, ("img", (9, 10, 8), 2), ["-c", "1"]), ("th2_err", 0, ("img", (12, 10, 9), 2), ["-c", "2"])]


@pytest.mark.parametrize("name,analysis,spec,flags", CASES)
def test_pcg3_fp64(tmp_path, name, analysis, spec, flags):
    nf, raw = build_small(tmp_path, name, analysis, spec)
    Cref, logref = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags)
    C, log = H.run_exec(H.CHFEM_EXEC, nf, raw, *flags, "-s", "2")
    assert H.rel_to_max(C, Cref) < FP64_TOL
    its, its_ref = H.parse_iterations(log), H.parse_iterations(logref)
    assert len(its) == len(its_ref) and all(abs(a - b) <= 1 for a, b in zip(its, its_ref)), (its, its_ref)


@pytest.mark.parametrize("name,analysis,spec,flags", CASES[:2])
def test_pcg3_mixed(tmp_path, name, analysis, spec, flags):
    nf, raw = build_small(tmp_path, name, analysis, spec)
    Cref, logref = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags)
    C, log = H.run_exec(H.CHFEM_EXEC, nf, raw, *flags, "-s", "2", "--precision", "mixed")
    assert H.rel_to_max(C, Cref) < MIXED_TOL
    assert_mixed_converges(log, logref)


def test_pcg3_initial_guess(tmp_path):
    """-xi with the 3-vector PCG: b - A x0 is formed in place in r (its only copy of b)."""
    nf, raw = build_small(tmp_path, "x3", 1, ("img", (8, 9, 10), 2))
    C1, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-d", "2", "-xo")
    C2, log = H.run_exec(H.CHFEM_EXEC, nf, raw, "-d", "2", "-s", "2", "-xi", nf[:-3] + "_X")
    assert "Initial guess satisfied" in log
    assert H.rel_to_max(C2[:, 2], C1[:, 2]) < 1e-12


def _bytes_per_dof(tmp_path, analysis, solver, precision):
    from chfem_b200 import _native
    img = H.small_image((16, 20, 18), 2, seed=zlib.crc32(b"mem") % 1000)
    nf, raw = H.write_small_case(str(tmp_path), f"m{analysis}{solver}{precision}", img, analysis, tol=1e-6)
    a = host_arrays(nf, raw)
    lib = _native.cudapcg()
    _native.setup_cudapcg_model(lib, a)
    assert lib.cudapcgSetSolver(solver)
    assert lib.cudapcgB200SetPrecision(precision)
    assert lib.cudapcgAllocateArrays()
    rhs = np.random.default_rng(1).standard_normal(a["ndof"])
    assert lib.cudapcgSetRHS(rhs.ctypes.data_as(ctypes.c_void_p))
    x = np.zeros(a["ndof"])
    lib.cudapcgSolve(x.ctypes.data_as(ctypes.c_void_p))
    assert not lib.cudapcgB200LastError(), lib.cudapcgB200LastError()
    maps = 2 * a["N"]  # the 16-bit node keys
    b = (lib.cudapcgB200DeviceBytes() - maps) / a["ndof"]
    lib.cudapcgEnd()
    return b


@pytest.mark.parametrize("analysis", [0, 1])
def test_device_bytes_per_unknown(tmp_path, analysis):
    assert _bytes_per_dof(tmp_path, analysis, 0, 0) <= 48  # PCG, FP64
    assert _bytes_per_dof(tmp_path, analysis, 2, 0) <= 32  # 3-vector PCG, FP64
    assert _bytes_per_dof(tmp_path, analysis, 2, 1) <= 36  # 3-vector PCG, mixed (x, b, r - A x scratch in FP64)
