"""Stokes DOF-number maps built on the device (cudapcgB200SetPoreImageColors) against the host
numbering (the reference's rule, femhmg_fluid_3D.c:370-491, restated in hmg_physics.cpp and
checked bit for bit against the reference's own host code in tests/test_host_parity.py):
node -> DOF, DOF -> node and the interface keys must be equal, element for element."""
import ctypes

import numpy as np
import pytest

from tests import helpers as H
from tests.test_gpu_parity import host_arrays

pytestmark = pytest.mark.gpu


def _device_maps(colors_zyx, refinement, pore_colour=0):
    from chfem_b200 import _native
    lib = _native.cudapcg()
    nz, ny, nx = colors_zyx.shape
    R, C, L = ny * refinement, nx * refinement, nz * refinement
    assert lib.cudapcgInit(5, 0)
    lib.cudapcgNewModel.restype = ctypes.POINTER(_native.CudapcgModel)
    m = lib.cudapcgNewModel()
    mm = m.contents
    mm.nrows, mm.ncols, mm.nlayers, mm.nelem = R, C, L, R * C * L
    mm.nvars, mm.nkeys, mm.localmtxdim, mm.poremap_flag = 1, 1, 1024, 1
    assert lib.cudapcgSetModel(m)
    lut = (ctypes.c_int * 256)(*[-1] * 256)
    for c in np.unique(colors_zyx):
        lut[int(c)] = 0 if int(c) == pore_colour else 1
    flat = np.ascontiguousarray(colors_zyx.reshape(-1))  # x fastest, as the .raw file
    nv, nb = ctypes.c_uint(), ctypes.c_uint()
    ok = lib.cudapcgB200SetPoreImageColors(flat.ctypes.data_as(ctypes.c_void_p), ny, nx, nz, refinement, lut,
                                           ctypes.byref(nv), ctypes.byref(nb))
    assert ok, lib.cudapcgB200LastError()
    N = R * C * L
    d2n = np.zeros(N, np.uint32)
    n2d = np.zeros(max(1, nv.value + nb.value), np.uint32)
    bk = np.zeros(max(1, nb.value), np.uint8)
    assert lib.cudapcgB200GetPoreMaps(d2n.ctypes.data_as(ctypes.c_void_p), n2d.ctypes.data_as(ctypes.c_void_p),
                                      bk.ctypes.data_as(ctypes.c_void_p))
    lib.cudapcgEnd()
    return nv.value, nb.value, d2n, n2d[: nv.value + nb.value], bk[: nb.value]


@pytest.mark.parametrize("shape,porosity,refinement", [((16, 18, 20), 0.45, 1), ((9, 7, 11), 0.5, 2), ((1, 12, 33), 0.6, 1),
                                                        ((160, 170, 180), 0.35, 1)])
def test_device_pore_maps_equal_host(tmp_path, shape, porosity, refinement):
    from chfem_b200.synthetic import pore_grf
    img = pore_grf(shape, corr=2.0, porosity=porosity, seed=17)
    nf, raw = H.write_small_case(str(tmp_path), "pm", img, 2, refinement=refinement)
    a = host_arrays(nf, raw)  # the host numbering
    nv, nb, d2n, n2d, bk = _device_maps(img, refinement)
    assert (nv, nb) == (a["nV"], a["nB"])
    assert np.array_equal(d2n, a["dof_of_node"])
    assert np.array_equal(n2d, a["node_of_dof"][: nv + nb])
    assert np.array_equal(bk, a["border"][:nb])
