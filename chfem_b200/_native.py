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
            "(python -m chfem_b200.build)")
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
        lib._typed = True
    return lib


class SolveStats(ctypes.Structure):
    """Mirror of chfemB200SolveStats (include/chfem_b200.h)."""
    _fields_ = [("n_cases", ctypes.c_int), ("direction", ctypes.c_int * 6),
                ("iterations", ctypes.c_uint * 6), ("residual", ctypes.c_double * 6),
                ("solve_seconds", ctypes.c_double * 6), ("rhs_seconds", ctypes.c_double),
                ("update_seconds", ctypes.c_double), ("total_seconds", ctypes.c_double),
                ("kernel_launches", ctypes.c_ulonglong), ("ndof", ctypes.c_uint)]


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
