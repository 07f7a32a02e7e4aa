"""The operator entry point that allocates nothing (cudapcgB200ApplyOperatorNoAlloc).

Callers that cannot allocate device memory -- embedders whose device memory belongs to their
own allocator, or loops that must not pay cudaMalloc's implicit synchronisation -- pass every
input and output as their own device buffer; the entry point keeps its scratch in a fixed
file-scope device array.  Its result must equal the regular operator entry point's
(cudapcgB200ApplyOperator, which manages its own buffers) within the FP64 operator tolerance
of the other GPU tests, on two calls in a row (the second call finds the array holding the
first call's leftovers).  Collected last, so a run stopped at its first failure has already
run every other test.
"""
import ctypes
import zlib

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu

OP_TOL = 1e-12  # relative to the largest entry, as in test_gpu_parity.test_operator_and_jacobi


def _dense(lcl, analysis, nmat):
    if analysis == 1:  # elastic: already dense 24x24 per material
        return lcl.copy()
    # thermal: expand the 40 stored non-zeros per material to 8x8 (zeros where nodes share an edge)
    drow = lambda k: -((k & 3) >> 1)
    dcol = lambda k: 1 if (k & 3) in (1, 2) else 0
    dlay = lambda k: k >> 2
    edge = lambda a, b: ((drow(a) != drow(b)) + (dcol(a) != dcol(b)) + (dlay(a) != dlay(b))) == 1
    out = np.zeros(64 * nmat)
    for m in range(nmat):
        p = 0
        for a in range(8):
            for b in range(8):
                if not edge(a, b):
                    out[64 * m + 8 * a + b] = lcl[40 * m + p]
                    p += 1
    return out


# the last case has more column tiles (35 x 263 of 32 x 8 nodes) than the array has reduction
# slots (8192): the persistent schedule gives each CTA several tiles
@pytest.mark.parametrize("analysis,shape,nmat", [(1, (9, 33, 10), 2), (0, (13, 35, 17), 3), (0, (1, 1100, 2100), 2)])
def test_no_alloc_matches_regular_entry_point(tmp_path, analysis, shape, nmat):
    import torch
    from chfem_b200 import _native
    from tests.test_gpu_parity import host_arrays

    name = f"na{analysis}"
    img = H.small_image(shape, nmat, seed=zlib.crc32(name.encode()) % 10000)
    nf, raw = H.write_small_case(str(tmp_path), name, img, analysis, tol=1e-8, maxit=100)
    a = host_arrays(nf, raw)
    lib = _native.cudapcg()
    # the regular entry point (allocates and owns its buffers)
    _native.setup_cudapcg_model(lib, a)
    assert lib.cudapcgB200SetPrecision(0)
    rng = np.random.default_rng(3)
    xs = [rng.standard_normal(a["ndof"]) for _ in range(2)]
    refs = []
    for x in xs:
        y = np.zeros(a["ndof"])
        assert lib.cudapcgB200ApplyOperator(x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p))
        refs.append(y)
    lib.cudapcgEnd()

    # the no-allocation entry point: every buffer belongs to the caller (here, torch)
    fn = lib.cudapcgB200ApplyOperatorNoAlloc
    fn.argtypes = [ctypes.c_int] + [ctypes.c_uint] * 4 + [ctypes.c_void_p] * 6
    fn.restype = ctypes.c_int
    dev = torch.device("cuda:0")
    keys = torch.from_numpy(a["keys"].astype(np.int16)).to(dev)
    Kd = torch.from_numpy(_dense(a["lcl"], analysis, a["nkeys"])).to(dev)
    y = torch.empty(a["ndof"], dtype=torch.float64, device=dev)
    vav = torch.empty(1, dtype=torch.float64, device=dev)
    for x, yref in zip(xs, refs):  # two calls in a row
        v = torch.from_numpy(x).to(dev)
        torch.cuda.synchronize()
        ok = fn(3 if analysis == 1 else 1, a["ny"], a["nx"], a["nz"], a["nkeys"], keys.data_ptr(), Kd.data_ptr(),
                v.data_ptr(), y.data_ptr(), vav.data_ptr(), None)
        assert ok == 1, lib.cudapcgB200LastError()
        torch.cuda.synchronize()
        yh = y.cpu().numpy()
        assert H.rel_to_max(yh, yref) < OP_TOL
        assert abs(vav.item() - float(x @ yref)) <= OP_TOL * abs(float(x @ yref)) * 10


def test_no_alloc_rejects_bad_input():
    """Argument errors are reported before any device work (the pointers here are never read)."""
    from chfem_b200 import _native
    lib = _native.cudapcg()
    fn = lib.cudapcgB200ApplyOperatorNoAlloc
    fn.argtypes = [ctypes.c_int] + [ctypes.c_uint] * 4 + [ctypes.c_void_p] * 6
    fn.restype = ctypes.c_int
    keys, kd, v, y, vav = (ctypes.c_void_p(1 << 40), ctypes.c_void_p(2 << 40), ctypes.c_void_p(3 << 40),
                           ctypes.c_void_p(4 << 40), ctypes.c_void_p(5 << 40))
    assert fn(3, 0x7fffffff, 8, 1, 2, keys, kd, v, y, vav, None) == 0
    assert b"dimension" in lib.cudapcgB200LastError()
    assert fn(3, 8, 8, 8, 2, keys, kd, v, v, vav, None) == 0  # in place: y == v
    assert b"overlap" in lib.cudapcgB200LastError()
    assert fn(3, 8, 8, 8, 2, keys, kd, v, ctypes.c_void_p((3 << 40) + 8), vav, None) == 0  # y inside v
    assert b"overlap" in lib.cudapcgB200LastError()
    assert fn(5, 8, 8, 8, 1, keys, kd, v, y, vav, None) == 0
    assert fn(3, 8, 8, 8, 7, keys, kd, v, y, vav, None) == 0
