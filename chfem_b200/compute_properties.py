"""compute_property: the Python entry point, with chfem's signature and checks.

Mirrors chfem/compute_properties.py:7-140: same arguments, defaults ('minres' for
permeability, 'cg' otherwise), validation and error messages; a temporary .nf file carries the
settings, the image is handed over flattened in C order, and the result is the list-of-rows
tensor (3x3 conductivity / permeability, 6x6 stiffness).  The solve runs in chfem_b200's
native host layer and GPU library.  Keyword-only extras (no counterpart in the reference):
precision='fp64'|'mixed', multirhs (all load cases as one block solve), initial_guess='learned'
(elasticity: the trained network's prediction of every load case's solution starts PCG; the
tolerance and so the tensor are unchanged).  output_fields=prefix writes, per load case, the
solution and its field as <prefix>_temperature|displacement|velocity_<case>.bin and
<prefix>_flux|stress|pressure_<case>.bin (read them with import_*_field_from_chfem), like
chfem_exec -e.  Elasticity with {phase: (young, poisson, alpha)} also returns the effective thermal
expansion (Voigt xx yy zz yz xz xy) as a seventh row, like the reference.
"""
import ctypes
import os
import tempfile

import numpy as np

from . import _native
from .io import export_for_chfem


def compute_property(property, array, mat_props=None, voxel_size=1e-6, solver=None, solver_tolerance=1e-6,
                     solver_maxiter=10000, precondition=True, type_of_rhs=0, refinement=1, direction='all',
                     output_fields=None, nf_filepath=None, *, precision='fp64', multirhs=False, initial_guess=None):
    properties = {'conductivity': 0, 'elasticity': 1, 'permeability': 2}
    if property not in properties:
        raise ValueError(f"Invalid property: {property}")
    analysis_type = properties[property]
    directions = {'x': 0, 'y': 1, 'z': 2, 'yz': 3, 'xz': 4, 'xy': 5, 'all': 6}
    if direction not in directions:
        raise ValueError(f"Invalid direction: {direction}")
    direction_int = directions[direction]
    # elasticity with (young, poisson, alpha): the effective thermal expansion is returned as one
    # more row (compute_properties.py:66-79 of chfem, chfem_wrapper.c:43-80)
    thermal_expansion = (mat_props is not None and analysis_type == 1 and
                         any(hasattr(p, '__len__') and len(p) == 3 for p in mat_props.values()))
    if thermal_expansion:
        if direction != 'all':
            raise ValueError(f"Invalid direction for thermal expansion analysis: {direction}. Must be \"all\".")
        for mat, props in mat_props.items():
            if len(props) < 3:
                raise ValueError(f"Invalid properties {props} for material {mat}. Expected thermal expansion coefficient.")
    output_fields_flag = 1 if output_fields is not None else 0
    if solver is None:
        solver = 'minres' if property == 'permeability' else 'cg'
    solvers = {'cg': 0, 'minres': 1, 'cg3': 2, 'minres3': 3, 'cg2': 4, 'minres2': 5}
    if solver not in solvers:
        raise ValueError(f"Invalid solver type: {solver}")
    if solver in ('cg2', 'minres2') and (output_fields_flag or property != 'permeability'):
        raise ValueError(f"Invalid solver type: {solver}. Two-vectors solvers do not produce fields to be exported, "
                         "nor are implemented for conductivy or elasticity analyses.")
    solver_type = solvers[solver]
    if precision not in ('fp64', 'mixed'):
        raise ValueError(f"Invalid precision: {precision}")

    tmp = None
    if nf_filepath is not None:
        if not os.path.exists(nf_filepath):
            raise ValueError(f"The file {nf_filepath} does not exist.")
        nf_filename = nf_filepath
    else:
        if mat_props is None and property != 'permeability':
            raise ValueError("Material properties must be provided, e.g. [(phase_id, cond),] for conductivity or "
                             "[(phase_id, young, poisson),] for elasticity.")
        if array.dtype != np.uint8:
            raise ValueError("Domain must be uint8 dtype.")
        if not (array == 0).any():  # the reference checks this for every property (compute_properties.py:105-107)
            raise ValueError("No fluid phase found in the domain.")
        if output_fields is None:
            tmp = tempfile.NamedTemporaryFile(delete=False, suffix=".nf")
        else:
            # the fields are written beside the .nf file: <output_fields>_temperature_<case>.bin, ...
            path, _ = os.path.split(output_fields)
            if path != '' and not os.path.exists(path):
                raise ValueError(f"Output fields directory {path} does not exist.")
            tmp = open(output_fields + ".nf", 'wb')
        export_for_chfem(None, array, analysis_type=analysis_type, mat_props=mat_props, voxel_size=voxel_size,
                         solver_type=solver_type, rhs_type=type_of_rhs, refinement=refinement, export_raw=False,
                         export_nf=True, solver_tolerance=solver_tolerance, solver_maxiter=solver_maxiter,
                         tmp_nf_file=tmp)
        nf_filename = tmp.name
    guesses = None
    if initial_guess not in (None, 'zero', 'learned'):
        raise ValueError(f"Invalid initial_guess: {initial_guess}")
    if initial_guess == 'learned':
        # the trained network's prediction of every load case's solution (elasticity only)
        if property != 'elasticity':
            raise ValueError("initial_guess='learned' is provided for elasticity")
        if mat_props is None:
            raise ValueError("initial_guess='learned' needs mat_props")
        if refinement != 1 or any(n % 8 for n in np.shape(array)):
            raise ValueError("initial_guess='learned' needs refinement 1 and every axis divisible by 8")
        from . import learned
        guesses = learned.device_guesses(learned.default_net(), array, mat_props)
    try:
        flat = np.ascontiguousarray(np.reshape(array, array.size), dtype=np.uint8)
        lib = _native.chfem()
        lib.chfemB200SetExportFields(output_fields_flag)
        if guesses is not None:
            P = ctypes.c_void_p * 6
            lib.chfemB200SetInitialGuesses(6, P(*[g.data_ptr() for g in guesses]), 1)
        C = np.zeros(36, dtype=np.float64)
        n = lib.chfemB200Run(flat.ctypes.data_as(ctypes.c_void_p), nf_filename.encode(), direction_int, solver_type,
                             int(bool(precondition)), 1 if precision == 'mixed' else 0, int(bool(multirhs)),
                             C.ctypes.data_as(ctypes.c_void_p))
        if n == 0:
            raise RuntimeError("chfem_b200 failed: " + lib.chfemB200LastError().decode())
        out = C[: n * n].reshape(n, n).tolist()
        if thermal_expansion:
            lib.hmgGetThermalExpansion.restype = ctypes.POINTER(ctypes.c_double)
            na = lib.hmgGetThermalExpansionDim()
            if na:
                out.append(lib.hmgGetThermalExpansion()[:na])
    finally:
        if tmp is not None:
            tmp.close()
            os.remove(tmp.name)
    return out
