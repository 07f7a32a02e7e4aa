"""Host model layer (libchfem_b200.so) versus the reference's own host code.

The reference's femhmg host code (compiled from its sources into oracle/_ref) hands its maps,
local matrices and right-hand sides over the cudapcg ABI to the CPU oracle, which records
them.  chfem_b200's own host layer must produce the same arrays: maps bit-exact, matrices and
RHS to round-off, and the same effective-tensor column from the same solution vector.
CPU only: no solve runs on a GPU here.
"""
import ctypes
import os
import tempfile
import zlib

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.skipif(not H.oracle_available(), reason="oracle/_ref not built (needs the reference tree)")


def host_arrays(nf, raw, direction):
    from chfem_b200 import _native
    lib = _native.chfem()
    lib.chfemB200SetQuiet(1)
    assert lib.hmgInit(nf.encode(), raw.encode(), None, None), lib.chfemB200LastError()
    info = (ctypes.c_uint * 9)()
    lib.chfemB200ModelInfo(info)
    out = {}
    dt = {0: np.uint16, 1: np.uint32, 2: np.uint32, 3: np.uint8, 4: np.float64, 6: np.uint16, 7: np.float64}
    for w, t in dt.items():
        nbytes = lib.chfemB200ModelArraySize(w)
        a = np.zeros(nbytes // np.dtype(t).itemsize, dtype=t)
        if nbytes:
            lib.chfemB200CopyModelArray(w, a.ctypes.data_as(ctypes.c_void_p), nbytes)
        out[w] = a
    ndof = info[4]
    rhs = np.zeros(ndof)
    lib.chfemB200AssembleRHS(direction, rhs.ctypes.data_as(ctypes.c_void_p))
    out["rhs"] = rhs
    out["info"] = list(info)
    return lib, out


def updateC(lib, direction, x):
    C = np.zeros(36)
    lib.chfemB200UpdateC(direction, np.ascontiguousarray(x).ctypes.data_as(ctypes.c_void_p), C.ctypes.data_as(ctypes.c_void_p))
    return C


CASES = [
    # name, analysis, shape (z,y,x), nmat, directions
    ("th2", 0, (6, 9, 11), 2, [0, 1, 2]),
    ("th4", 0, (5, 7, 4), 4, [0, 2]),
    ("el2", 1, (5, 6, 7), 2, [0, 1, 2, 3, 4, 5]),
    ("el3", 1, (4, 5, 3), 3, [1, 3, 5]),
]


@pytest.mark.parametrize("name,analysis,shape,nmat,dirs", CASES)
def test_thermal_elastic_maps_rhs_updateC(tmp_path, name, analysis, shape, nmat, dirs):
    img = H.small_image(shape, nmat, seed=zlib.crc32(name.encode()) % 1000)
    nf, raw = H.write_small_case(str(tmp_path), name, img, analysis, tol=1e-6, maxit=50)
    for d in dirs:
        ref = H.oracle_capture(nf, raw, d)
        lib, mine = host_arrays(nf, raw, d)
        assert np.array_equal(mine[0], ref["0"]), "node material keys differ"
        np.testing.assert_allclose(mine[4], ref["4"], rtol=1e-12, atol=1e-12 * np.abs(ref["4"]).max())
        np.testing.assert_allclose(mine["rhs"], ref["5"], rtol=1e-11, atol=1e-11 * np.abs(ref["5"]).max())
        C = updateC(lib, d, ref["6"])
        k = 6 if analysis == 1 else 3
        col_mine = C[: k * k].reshape(k, k)[:, d]
        col_ref = ref["C"][: k * k].reshape(k, k)[:, d]
        assert H.rel_to_max(col_mine, col_ref) < 1e-12


CASES_2D = [
    # name, analysis, shape (y, x), nmat, directions (2D elastic: X, Y, XY = 0, 1, 5)
    ("th2d2", 0, (9, 11), 2, [0, 1]),
    ("th2d4", 0, (6, 5), 4, [1]),
    ("el2d2", 1, (7, 10), 2, [0, 1, 5]),
    ("el2d3", 1, (5, 4), 3, [5]),
]


@pytest.mark.parametrize("name,analysis,shape,nmat,dirs", CASES_2D)
def test_2d_maps_rhs_updateC(tmp_path, name, analysis, shape, nmat, dirs):
    """2D pixel models (femhmg_2D.c, femhmg_thermal_2D.c, femhmg_elastic_2D.c): 4-bit node keys
    bit-exact, element matrices (dense 4x4 / 8x8, plane strain) and right-hand sides to round-off,
    the tensor column from the reference's solution vector."""
    img = H.small_image(shape, nmat, seed=zlib.crc32(name.encode()) % 1000)
    nf, raw = H.write_small_case(str(tmp_path), name, img, analysis, tol=1e-6, maxit=50)
    for d in dirs:
        ref = H.oracle_capture(nf, raw, d)
        lib, mine = host_arrays(nf, raw, d)
        assert mine["info"][2] == 1
        assert np.array_equal(mine[0], ref["0"]), "node material keys differ"
        np.testing.assert_allclose(mine[4], ref["4"], rtol=1e-12, atol=1e-12 * np.abs(ref["4"]).max())
        np.testing.assert_allclose(mine["rhs"], ref["5"], rtol=1e-11, atol=1e-11 * np.abs(ref["5"]).max())
        C = updateC(lib, d, ref["6"])
        k = 3 if analysis == 1 else 2
        col = 2 if d == 5 else d
        assert H.rel_to_max(C[: k * k].reshape(k, k)[:, col], ref["C"][: k * k].reshape(k, k)[:, col]) < 1e-12


def test_fluid_maps_rhs_updateC(tmp_path):
    from chfem_b200.synthetic import pore_grf
    img = pore_grf((10, 12, 14), corr=2.0, porosity=0.45, seed=7)
    assert (img == 0).any()
    nf, raw = H.write_small_case(str(tmp_path), "fl", img, 2, tol=1e-6, maxit=50)
    for d in [0, 1, 2]:
        ref = H.oracle_capture(nf, raw, d)
        lib, mine = host_arrays(nf, raw, d)
        assert np.array_equal(mine[1], ref["1"]), "node->DOF map differs"
        assert np.array_equal(mine[2], ref["2"]), "DOF->node map differs"
        assert np.array_equal(mine[3], ref["3"]), "interface fluid keys differ"
        np.testing.assert_allclose(mine[4], ref["4"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(mine["rhs"], ref["5"], rtol=1e-12, atol=1e-14)
        C = updateC(lib, d, ref["6"])
        assert H.rel_to_max(C[:9].reshape(3, 3)[:, d], ref["C"][:9].reshape(3, 3)[:, d]) < 1e-12


def test_fluid_2d_maps_rhs_updateC(tmp_path):
    """2D Stokes (femhmg_fluid_2D.c): fluid keys, DOF numbering (pore nodes first, then interface
    nodes), DOF->node map and interface keys bit-exact; the 12 x 12 element matrix, right-hand
    sides and permeability column equal the reference's host code."""
    rng = np.random.default_rng(21)
    img = np.where(rng.random((14, 17)) < 0.3, 255, 0).astype(np.uint8)
    nf, raw = H.write_small_case(str(tmp_path), "fl2d", img, 2, tol=1e-6, maxit=50)
    for d in [0, 1]:
        ref = H.oracle_capture(nf, raw, d)
        lib, mine = host_arrays(nf, raw, d)
        assert np.array_equal(mine[1], ref["1"]), "node->DOF map differs"
        assert np.array_equal(mine[2], ref["2"]), "DOF->node map differs"
        assert np.array_equal(mine[3], ref["3"]), "interface fluid keys differ"
        np.testing.assert_allclose(mine[4], ref["4"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(mine["rhs"], ref["5"], rtol=1e-12, atol=1e-14)
        C = updateC(lib, d, ref["6"])
        assert H.rel_to_max(C[:4].reshape(2, 2)[:, d], ref["C"][:4].reshape(2, 2)[:, d]) < 1e-12


def test_refinement_and_transpose(tmp_path):
    """%refinement replicates each voxel and the x-fastest file order is transposed."""
    img = H.small_image((3, 4, 5), 2, seed=3)
    nf, raw = H.write_small_case(str(tmp_path), "ref2", img, 0, tol=1e-6, maxit=50, refinement=2)
    ref = H.oracle_capture(nf, raw, 0)
    lib, mine = host_arrays(nf, raw, 0)
    assert mine["info"][:3] == [10, 8, 6]
    assert np.array_equal(mine[0], ref["0"])
    np.testing.assert_allclose(mine["rhs"], ref["5"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name,shape", [("te3d", (5, 6, 7)), ("te2d", (9, 12))])
def test_thermal_expansion_rhs(tmp_path, name, shape):
    """The thermal-expansion load (a unit temperature rise; femhmg_elastic_3D.c:464-505,
    femhmg_elastic_2D.c:277-300): the reference's host code hands it over last (after the load
    case), chfem_b200's host layer assembles the same vector."""
    from chfem_b200 import _native
    from tests.test_thermal_expansion import write_case
    img = H.small_image(shape, 2, seed=zlib.crc32(name.encode()) % 1000)
    nf, raw = write_case(tmp_path, name, img, {0: (1.0, 0.3, 2e-5), 255: (10.0, 0.2, -1e-5)})
    ref = H.oracle_capture(nf, raw, 0)
    lib, mine = host_arrays(nf, raw, 0)
    rhs = np.zeros(mine["info"][4])
    assert lib.chfemB200AssembleThermalExpansionRHS(rhs.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_allclose(rhs, ref["5"], rtol=1e-11, atol=1e-11 * np.abs(ref["5"]).max())
    assert np.abs(rhs).max() > 0


@pytest.mark.parametrize("name,shape", [("tu3d", (5, 6, 7)), ("tu2d", (9, 12))])
def test_thermal_expansion_update(tmp_path, name, shape):
    """The effective thermal expansion from the reference's own solution of the unit-temperature
    load and its own tensor (all load cases, femhmg_elastic_3D.c:863-1074,
    femhmg_elastic_2D.c:388-528): chfem_b200's host layer returns the reference's coefficients."""
    from tests.test_thermal_expansion import write_case
    img = H.small_image(shape, 2, seed=zlib.crc32(name.encode()) % 1000)
    nf, raw = write_case(tmp_path, name, img, {0: (1.0, 0.3, 2e-5), 255: (10.0, 0.2, -1e-5)})
    ref = H.oracle_capture(nf, raw, 6)  # every load case, then the thermal-expansion solve
    lib, mine = host_arrays(nf, raw, 0)
    na = 3 if len(shape) == 2 else 6
    alpha = np.zeros(na)
    x = np.ascontiguousarray(ref["6"])
    C = np.ascontiguousarray(ref["C"])
    assert lib.chfemB200UpdateThermalExpansion(x.ctypes.data_as(ctypes.c_void_p), C.ctypes.data_as(ctypes.c_void_p),
                                               alpha.ctypes.data_as(ctypes.c_void_p))
    assert ref["alpha"].size == na
    assert H.rel_to_max(alpha, ref["alpha"]) < 1e-9, (alpha, ref["alpha"])
