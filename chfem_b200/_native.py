"""Loaders for the chfem_b200 native libraries (built in-tree under chfem_b200/lib/).

The product path is native: libcudapcg_b200.so runs the solver on the GPU and
libchfem_b200.so is the host model layer.  A missing library is an error, never a silent
fallback to another implementation.
"""
import ctypes
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
_libs = {}


class NativeLibraryMissing(RuntimeError):
    pass


def lib_path(name):
    return os.path.join(LIB_DIR, name)


def _load(name):
    if name in _libs:
        return _libs[name]
    path = lib_path(name)
    if not os.path.exists(path):
        raise NativeLibraryMissing(
            f"{path} is missing: build the chfem_b200 native libraries first "
            "(python -c 'import __graft_entry__; __graft_entry__.build()' at the repository root)")
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    _libs[name] = lib
    return lib


def cudapcg():
    """The GPU solver library (drop-in cudapcg C ABI + cudapcgB200* extensions)."""
    lib = _load("libcudapcg_b200.so")
    if not getattr(lib, "_typed", False):
        c = ctypes
        lib.cudapcgB200LastError.restype = c.c_char_p
        lib.cudapcgB200TimeOperator.restype = c.c_double
        lib.cudapcgB200TimeOperator.argtypes = [c.c_uint]
        lib.cudapcgB200DeviceBytes.restype = c.c_ulonglong
        lib.cudapcgGetResidual.restype = c.c_double
        lib.cudapcgSetNumTol.argtypes = [c.c_double]
        lib.cudapcgB200SetImageColors.restype = c.c_ubyte
        lib.cudapcgB200SetImageColors.argtypes = [c.c_void_p, c.c_uint, c.c_uint, c.c_uint, c.c_uint, c.c_void_p]
        lib._typed = True
    return lib


def chfem():
    """The host model layer (femhmg-compatible hmg* API + chfemB200* extensions)."""
    cudapcg()  # dependency first, so its loader typing is in place
    lib = _load("libchfem_b200.so")
    if not getattr(lib, "_typed", False):
        c = ctypes
        lib.hmgInit.argtypes = [c.c_char_p, c.c_char_p, c.c_char_p, c.c_void_p]
        lib.hmgInit.restype = c.c_uint8
        lib.hmgGetConstitutiveMtx.restype = c.POINTER(c.c_double)
        lib.hmgGetConstitutiveMtxDim.restype = c.c_uint
        lib.chfemB200LastError.restype = c.c_char_p
        lib.chfemB200ModelArraySize.restype = c.c_ulonglong
        lib.chfemB200ModelArraySize.argtypes = [c.c_int]
        lib.chfemB200CopyModelArray.argtypes = [c.c_int, c.c_void_p, c.c_ulonglong]
        lib.chfemB200AssembleRHS.argtypes = [c.c_int, c.c_void_p]
        lib.chfemB200UpdateC.argtypes = [c.c_int, c.c_void_p, c.c_void_p]
        lib.chfemB200Run.argtypes = [c.c_void_p, c.c_char_p, c.c_int, c.c_int, c.c_int, c.c_int, c.c_int, c.c_void_p]
        lib.chfemB200Run.restype = c.c_int
        lib.chfemB200SetExportFields.argtypes = [c.c_int]
        lib.chfemB200RunThermalBatch.argtypes = [c.c_uint, c.c_void_p, c.c_double, c.c_uint, c.c_int, c.c_void_p, c.c_void_p,
                                                 c.c_void_p]
        lib.chfemB200RunThermalBatch.restype = c.c_int
        lib._typed = True
    return lib


class BatchStats(ctypes.Structure):
    """Mirror of cudapcgB200BatchStats (include/cudapcg_b200.h)."""
    _fields_ = [("setup_seconds", ctypes.c_double), ("solve_seconds", ctypes.c_double), ("wall_seconds", ctypes.c_double),
                ("max_iterations", ctypes.c_uint), ("converged", ctypes.c_uint), ("kernel_launches", ctypes.c_ulonglong),
                ("tile_cols", ctypes.c_int), ("ctas_operator", ctypes.c_int), ("ctas_pointwise", ctypes.c_int),
                ("tile_ms", ctypes.c_double * 3)]


def batch_stats():
    st = BatchStats()
    chfem().chfemB200LastBatchStats(ctypes.byref(st))
    return st


class ThermalSample(ctypes.Structure):
    """Mirror of chfemB200ThermalSample (include/chfem_b200.h)."""
    _fields_ = [("nx", ctypes.c_uint), ("ny", ctypes.c_uint), ("nz", ctypes.c_uint), ("voxels", ctypes.c_void_p),
                ("nmat", ctypes.c_uint), ("colors", ctypes.c_uint8 * 4), ("conductivity", ctypes.c_double * 4)]


class SolveStats(ctypes.Structure):
    """Mirror of chfemB200SolveStats (include/chfem_b200.h)."""
    _fields_ = [("n_cases", ctypes.c_int), ("direction", ctypes.c_int * 6),
                ("iterations", ctypes.c_uint * 6), ("residual", ctypes.c_double * 6),
                ("solve_seconds", ctypes.c_double * 6), ("rhs_seconds", ctypes.c_double),
                ("update_seconds", ctypes.c_double), ("total_seconds", ctypes.c_double),
                ("kernel_launches", ctypes.c_ulonglong), ("ndof", ctypes.c_uint), ("setup_seconds", ctypes.c_double),
                ("solve_call_seconds", ctypes.c_double), ("teardown_seconds", ctypes.c_double)]


class CudapcgStats(ctypes.Structure):
    """Mirror of cudapcgB200Stats (include/cudapcg_b200.h)."""
    _fields_ = [("iterations", ctypes.c_uint), ("residual", ctypes.c_double),
                ("solve_seconds", ctypes.c_double), ("setup_seconds", ctypes.c_double),
                ("kernel_launches", ctypes.c_ulonglong), ("precision", ctypes.c_int),
                ("found", ctypes.c_int)]


def solve_stats():
    st = SolveStats()
    chfem().chfemB200GetSolveStats(ctypes.byref(st))
    return st


class CudapcgModel(ctypes.Structure):
    """Mirror of cudapcgModel_t (include/cudapcg_b200.h; chfem/src/femhmg/cudapcg/includes.h:93-129)."""
    _fields_ = [("name", ctypes.c_char_p), ("freeAllowed_flag", ctypes.c_uint8), ("parStrategy_flag", ctypes.c_uint8),
                ("poremap_flag", ctypes.c_uint8), ("parametric_density_field_flag", ctypes.c_uint8), ("SBS_flag", ctypes.c_uint8),
                ("nrows", ctypes.c_uint), ("ncols", ctypes.c_uint), ("nlayers", ctypes.c_uint), ("nelem", ctypes.c_uint),
                ("nvars", ctypes.c_uint), ("nvarspernode", ctypes.c_uint), ("nkeys", ctypes.c_uint), ("localmtxdim", ctypes.c_uint),
                ("nporenodes", ctypes.c_uint), ("nbordernodes", ctypes.c_uint), ("nhmgvars", ctypes.c_uint),
                ("limits_density_field", ctypes.c_double * 2), ("image", ctypes.c_void_p), ("parametric_density_field", ctypes.c_void_p),
                ("pore_map", ctypes.c_void_p), ("border_pore_map", ctypes.c_void_p), ("periodic2DOF_map", ctypes.c_void_p),
                ("DOF2periodic_map", ctypes.c_void_p)]


def setup_cudapcg_model(lib, arrays):
    """Drive the cudapcg C ABI of `lib` with host-layer arrays: init, model, maps, local matrices.

    arrays: dict with nx, ny, nz, N, ndof, nV, nB, nkeys, analysis (0/1/2), keys, dof_of_node,
    node_of_dof, border, lcl (the formats of the cudapcg ABI)."""
    a = arrays
    an = {0: 1, 1: 3, 2: 5}[a["analysis"]]
    assert lib.cudapcgInit(an, 0)
    lib.cudapcgNewModel.restype = ctypes.POINTER(CudapcgModel)
    m = lib.cudapcgNewModel()
    mm = m.contents
    mm.nrows, mm.ncols, mm.nlayers = a["ny"], a["nx"], a["nz"]
    mm.nelem = a["N"]
    mm.nvars = a["ndof"]
    mm.nkeys = a["nkeys"]
    mm.localmtxdim = a["lcl"].size // a["nkeys"]
    mm.nporenodes, mm.nbordernodes = a["nV"], a["nB"]
    mm.nhmgvars = 3 * a["nV"] if a["analysis"] == 2 else a["ndof"]
    mm.poremap_flag = 1
    assert lib.cudapcgSetModel(m)
    import numpy as np
    keep = []

    def ptr(x):
        x = np.ascontiguousarray(x)
        keep.append(x)
        return x.ctypes.data_as(ctypes.c_void_p)
    if a["analysis"] == 2:
        assert lib.cudapcgSetPeriodic2DOFMap(ptr(a["dof_of_node"]))
        assert lib.cudapcgSetPoreMap(ptr(a["border"]))
        assert lib.cudapcgSetDOF2PeriodicMap(ptr(a["node_of_dof"]))
    else:
        assert lib.cudapcgSetImage(ptr(a["keys"]))
    assert lib.cudapcgSetLclMtxs(ptr(a["lcl"]))
