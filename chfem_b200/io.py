"""chfem input/output formats: the .nf settings file and the .raw voxel image.

Same functions, arguments and file formats as chfem's Python I/O (chfem/io.py:3-109 import_nf,
import_raw; :208-335 export_for_chfem).  A .raw image is the uint8 voxel array in C order of a
(z, y, x) array, i.e. x fastest; the .nf file is a list of '%tag' lines each followed by its
values.
"""
import numpy as np


def import_nf(filename):
    """Read a .nf file into a dict (keys as in chfem/io.py:3-71).

    image_dimensions is returned as (nz, ny, nx) for numpy indexing of the image.
    """
    if not filename.endswith(".nf"):
        raise ValueError("Filename does not end with '.nf'")
    with open(filename) as f:
        lines = [ln.rstrip() for ln in f]
    data = {}
    for key in ("type_of_analysis", "type_of_solver", "type_of_rhs", "number_of_iterations", "refinement",
                "number_of_materials"):
        data[key] = int(lines[lines.index(f"%{key}") + 1])
    data["voxel_size"] = float(lines[lines.index("%voxel_size") + 1])
    data["solver_tolerance"] = float(lines[lines.index("%solver_tolerance") + 1])
    nx, ny, nz = (int(v) for v in lines[lines.index("%image_dimensions") + 1].split())
    data["image_dimensions"] = (nz, ny, nx)
    i = lines.index("%properties_of_materials")
    data["properties_of_materials"] = []
    for j in range(1, data["number_of_materials"] + 1):
        parts = lines[i + j].split()
        data["properties_of_materials"].append((int(parts[0]), *[float(p) for p in parts[1:]]))
    data["volume_fraction"] = None
    if "%volume_fraction" in lines:
        data["volume_fraction"] = tuple(float(v) for v in lines[lines.index("%volume_fraction") + 1].split())
    data["data_type"] = None
    if "%data_type" in lines:
        data["data_type"] = lines[lines.index("%data_type") + 1]
    if "%thermal_expansion" in lines:
        i = lines.index("%thermal_expansion")
        data["thermal_expansion"] = [float(lines[i + j]) for j in range(1, data["number_of_materials"] + 1)]
    return data


def import_raw(filename, shape=None, dtype=np.uint8):
    """Read a .raw file into a numpy array; shape is (z, y, x) for 3D (chfem/io.py:73-109)."""
    if not filename.endswith(".raw"):
        raise ValueError("Filename does not end with '.raw'")
    with open(filename, "rb") as f:
        raw = f.read()
    if shape is not None:
        expected = int(np.prod(shape)) * np.dtype(dtype).itemsize
        if len(raw) != expected:
            raise ValueError(f"File size ({len(raw)}) does not match expected size ({expected})")
    arr = np.frombuffer(raw, dtype=dtype)
    return arr.reshape(shape) if shape is not None else arr


def export_for_chfem(filename, array, analysis_type, mat_props=None, voxel_size=1, solver_type=0, rhs_type=0,
                     refinement=1, export_raw=True, export_nf=True, solver_tolerance=1.e-6, solver_maxiter=10000,
                     tmp_nf_file=None):
    """Write the .nf (and optionally .raw) inputs of an analysis (chfem/io.py:208-335).

    analysis_type: 0 conductivity ({phase: k}), 1 elasticity ({phase: (E, nu[, alpha])}),
    2 permeability (mat_props None).  Returns the dict of written settings.
    """
    domain = array.astype(np.uint8)
    hist = np.bincount(domain.reshape(-1), minlength=256)  # voxels per colour (a sort-free count)
    ids = np.nonzero(hist)[0]
    materials = dict(zip(ids.tolist(), hist[ids].tolist()))
    if mat_props is not None:
        props_ids, img_ids = set(mat_props.keys()), set(materials.keys())
        if props_ids != img_ids:
            msg = []
            if img_ids - props_ids:
                msg.append(f"Missing material IDs in 'mat_props' that are present in the array: {img_ids - props_ids}.")
            if props_ids - img_ids:
                msg.append(f"Extra material IDs in 'mat_props' that are not present in the array: {props_ids - img_ids}.")
            raise ValueError(" ".join(msg))
    props, alphas = [], []
    if analysis_type == 0:
        props = [f"{k} {v}" for k, v in mat_props.items()]
    elif analysis_type == 1:
        for k, v in mat_props.items():
            props.append(f"{k} {v[0]} {v[1]}")
            if len(v) == 3:
                alphas.append(f"{v[2]}")
            elif alphas:
                alphas.append("0.0")
    elif analysis_type == 2:
        props = [f"{k}" for k in materials.keys()]
    else:
        raise ValueError("Invalid analysis type.")
    vf = np.array(list(materials.values())) * 100.0 / np.prod(domain.shape)
    dims = [domain.shape[1], domain.shape[0], 0] if domain.ndim == 2 else [domain.shape[2], domain.shape[1], domain.shape[0]]
    jdata = {"type_of_analysis": analysis_type, "type_of_solver": solver_type, "type_of_rhs": rhs_type,
             "voxel_size": voxel_size, "solver_tolerance": solver_tolerance, "number_of_iterations": solver_maxiter,
             "image_dimensions": dims, "refinement": refinement, "number_of_materials": len(materials),
             "properties_of_materials": props, "volume_fraction": list(np.around(vf, 2)), "data_type": "uint8"}
    if alphas:
        jdata["thermal_expansion"] = alphas
    if export_nf:
        out = []
        for k, v in jdata.items():
            out.append("%" + k)
            if k in ("properties_of_materials", "thermal_expansion"):
                out.extend(v)
            elif isinstance(v, (list, tuple)):
                out.append(" ".join(str(float(x)) if isinstance(x, (np.floating,)) else str(x) for x in v))
            else:
                out.append(str(v))
            out.append("")
        text = "\n".join(out).strip()
        if tmp_nf_file is not None:
            tmp_nf_file.write(text.encode("utf-8"))
            tmp_nf_file.flush()
            tmp_nf_file.seek(0)
        else:
            with open(filename[: len(filename) - 4] + ".nf", "w") as f:
                f.write(text)
    if export_raw:
        fn = filename if filename.endswith(".raw") else filename + ".raw"
        domain.tofile(fn)
    return jdata


# ---- exported fields (-e / compute_property(output_fields=...)) ------------------------------
# A field file holds float64 node values with the row index fastest, then column, then layer
# (node = row + col*ny + layer*ny*nx) and the per-node components innermost: a C-order
# [z][x][y](, k) array.  The readers below hand it back as [z][y][x] (image order) or, with
# rotate_domain, as [x][y][z]; the component axis comes first.  Same functions, arguments and
# results as chfem/io.py:111-206 (3D; 2D fields are stored [x][y](, k)).

def _read_field(filename, domain_shape, ncomp, rotate_domain, dtype):
    data = np.fromfile(filename, dtype=dtype)
    if len(domain_shape) == 2:
        ny, nx = domain_shape
        a = data.reshape((nx, ny) + ((ncomp,) if ncomp else ()))
        if ncomp:
            return a.transpose(2, 0, 1) if rotate_domain else a.transpose(2, 1, 0)
        return a if rotate_domain else a.T
    nz, ny, nx = domain_shape
    a = data.reshape((nz, nx, ny) + ((ncomp,) if ncomp else ()))
    if ncomp:
        return a.transpose(3, 1, 2, 0) if rotate_domain else a.transpose(3, 0, 2, 1)
    return a.transpose(1, 2, 0) if rotate_domain else a.transpose(0, 2, 1)


def import_scalar_field_from_chfem(filename, domain_shape, rotate_domain=False, dtype=np.float64):
    """Scalar node field (temperature, pressure) of an image of shape domain_shape ((nz, ny, nx)
    or (ny, nx)); returned as [z][y][x] ([y][x]), or [x][y][z] ([x][y]) with rotate_domain."""
    return _read_field(filename, domain_shape, 0, rotate_domain, dtype)


def import_vector_field_from_chfem(filename, domain_shape, rotate_domain=False, dtype=np.float64):
    """Vector node field (flux, displacement, velocity): [k][z][y][x] with k = 3 (2 in 2D), or
    [k][x][y][z] with rotate_domain."""
    return _read_field(filename, domain_shape, 2 if len(domain_shape) == 2 else 3, rotate_domain, dtype)


def import_stress_field_from_chfem(filename, domain_shape, rotate_domain=False, dtype=np.float64):
    """Stress node field: [k][z][y][x] with k = 6 Voigt components xx yy zz yz xz xy (3 in 2D),
    or [k][x][y][z] with rotate_domain."""
    return _read_field(filename, domain_shape, 3 if len(domain_shape) == 2 else 6, rotate_domain, dtype)
