"""Batched homogenization: many independent images solved together on the GPU.

The reference (and compute_property) homogenizes one image per call.  For many small images
the GPU is mostly idle in such a loop; compute_conductivity_batch solves all samples and their
3 load cases in one device-resident loop (chfemB200RunThermalBatch ->
cudapcgB200SolveThermalBatch), each load case with its own PCG scalars and stopping test, so
every tensor is the one compute_property returns for that image.
"""
import ctypes

import numpy as np

from . import _native


def compute_conductivity_batch(arrays, mat_props, solver_tolerance=1e-6, solver_maxiter=10000, precision="fp64",
                               return_iterations=False):
    """Effective conductivity tensors of many images.

    arrays: sequence of 3D uint8 arrays indexed (z, y, x), each any size;
    mat_props: one dict {colour: conductivity} for all samples, or a sequence of such dicts,
      one per sample (at most 4 colours each);
    precision: 'fp64' or 'mixed' (FP32 fields; FP64 solution, dots and residual replacement).
    Returns an (n, 3, 3) array (and the (n, 3) iteration counts with return_iterations).
    """
    arrays = [np.ascontiguousarray(a, dtype=np.uint8) for a in arrays]
    n = len(arrays)
    if n == 0:
        raise ValueError("no images")
    props = list(mat_props) if not isinstance(mat_props, dict) else [mat_props] * n
    if len(props) != n:
        raise ValueError("mat_props: one dict, or one per image")
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"Invalid precision: {precision}")
    samples = (_native.ThermalSample * n)()
    for s, (a, p) in enumerate(zip(arrays, props)):
        if a.ndim != 3:
            raise ValueError("each image must be a 3D (z, y, x) array")
        if not 1 <= len(p) <= 4:
            raise ValueError("1 to 4 materials per image")
        present = set(np.unique(a).tolist())
        missing = present - set(int(c) for c in p)
        if missing:
            raise ValueError(f"image {s}: colours {sorted(missing)} have no conductivity")
        t = samples[s]
        t.nz, t.ny, t.nx = a.shape
        t.voxels = a.ctypes.data
        t.nmat = len(p)
        for k, (c, kv) in enumerate(sorted(p.items())):
            t.colors[k] = int(c)
            t.conductivity[k] = float(kv)
    C = np.zeros((n, 9))
    its = np.zeros((n, 3), dtype=np.uint32)
    secs = ctypes.c_double(0.0)
    lib = _native.chfem()
    rc = lib.chfemB200RunThermalBatch(n, ctypes.cast(samples, ctypes.c_void_p), float(solver_tolerance), int(solver_maxiter),
                                      1 if precision == "mixed" else 0, C.ctypes.data, its.ctypes.data, ctypes.byref(secs))
    if rc == 0:
        raise RuntimeError(lib.chfemB200LastError().decode())
    C = C.reshape(n, 3, 3)
    return (C, its) if return_iterations else C
