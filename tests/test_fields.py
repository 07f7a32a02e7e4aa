"""Exported node fields (chfem_exec -e, compute_property(output_fields=...)).

CPU: the NumPy field oracle (oracle/fields_oracle.py) is pinned against the reference's own
saveFields code run through the oracle executable (reference host code + CPU solver), and the
field readers are checked on known layouts.  GPU: chfem_b200's solutions and fields, single
and block (--multirhs) solves, thermal / elastic / Stokes, against the oracle.
"""
import glob
import os
import sys
import zlib

import numpy as np
import pytest

from tests import helpers as H

sys.path.insert(0, os.path.join(H.ROOT, "oracle"))
import fields_oracle as FO  # noqa: E402

from chfem_b200 import io as cio  # noqa: E402

# The reference's saveFields loops run under OpenMP with unsynchronised += into shared nodes;
# one thread keeps its output deterministic.
ONE_THREAD = {"OMP_NUM_THREADS": "1"}
CASE_FILES = {0: ("temperature", "flux", 1, 3), 1: ("displacement", "stress", 3, 6)}


def _case(tmp_path, name, analysis, shape, nmat, refinement=1):
    img = H.small_image(shape, nmat, seed=zlib.crc32(name.encode()) % 10000)
    nf, raw = H.write_small_case(str(tmp_path), name, img, analysis, tol=1e-10, maxit=20000, refinement=refinement)
    return img, nf, raw


def _mats_and_props(nf, img, refinement):
    d = cio.import_nf(nf)
    codes = [p[0] for p in d["properties_of_materials"]]
    props = [p[1] if d["type_of_analysis"] == 0 else (p[1], p[2]) for p in d["properties_of_materials"]]
    return FO.materials_from_image(img, codes, refinement), props


def _load_case(direction, analysis):
    if analysis == 0:
        return direction, 0
    return {0: (0, 0), 1: (1, 1), 2: (2, 2), 3: (1, 2), 4: (2, 0), 5: (1, 0)}[direction]


def _check_fields_against_oracle(prefix, img, nf, analysis, refinement, rtol):
    sol, fld, nd, nfc = CASE_FILES[analysis]
    mat, props = _mats_and_props(nf, img, refinement)
    ndirs = 3 if analysis == 0 else 6
    for d in range(ndirs):
        x = np.fromfile(f"{prefix}_{sol}_{d}.bin")
        f = np.fromfile(f"{prefix}_{fld}_{d}.bin")
        assert x.size == mat.size * nd and f.size == mat.size * nfc
        axis, comp = _load_case(d, analysis)
        ref = FO.node_fields(x, mat, props, axis, comp, nd)
        assert H.rel_to_max(f, ref) < rtol, (d, H.rel_to_max(f, ref))


# ---- CPU: pin the field oracle on the reference's own saveFields ------------------------
needs_oracle = pytest.mark.skipif(not H.oracle_available(), reason="oracle executable not built")


@needs_oracle
@pytest.mark.parametrize("name,analysis,shape,nmat,refinement", [
    ("fth3", 0, (4, 5, 6), 3, 1),
    ("fel2", 1, (5, 4, 6), 2, 1),
    ("fth2_ref2", 0, (3, 2, 4), 2, 2),
])
def test_field_oracle_matches_reference_savefields(tmp_path, name, analysis, shape, nmat, refinement):
    img, nf, raw = _case(tmp_path, name, analysis, shape, nmat, refinement)
    H.run_exec(H.ORACLE_EXEC, nf, raw, "-e", env=ONE_THREAD)
    _check_fields_against_oracle(nf[:-3], img, nf, analysis, refinement, 1e-12)


def test_field_readers_layout(tmp_path):
    nz, ny, nx = 3, 4, 5
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    scal = 100 * z + 10 * y + x  # [z][y][x]
    # files hold the row (y) index fastest, then x, then z: a C-order [z][x][y] array
    scal.transpose(0, 2, 1).astype(np.float64).tofile(tmp_path / "s.bin")
    np.testing.assert_array_equal(cio.import_scalar_field_from_chfem(str(tmp_path / "s.bin"), (nz, ny, nx)), scal)
    np.testing.assert_array_equal(cio.import_scalar_field_from_chfem(str(tmp_path / "s.bin"), (nz, ny, nx), True),
                                  scal.transpose(2, 1, 0))
    vec = np.stack([scal + 1000 * k for k in range(6)])  # [k][z][y][x]
    vec.transpose(1, 3, 2, 0).astype(np.float64).tofile(tmp_path / "v.bin")
    np.testing.assert_array_equal(cio.import_stress_field_from_chfem(str(tmp_path / "v.bin"), (nz, ny, nx)), vec)
    np.testing.assert_array_equal(cio.import_stress_field_from_chfem(str(tmp_path / "v.bin"), (nz, ny, nx), True),
                                  vec.transpose(0, 3, 2, 1))
    vec[:3].transpose(1, 3, 2, 0).astype(np.float64).tofile(tmp_path / "w.bin")
    np.testing.assert_array_equal(cio.import_vector_field_from_chfem(str(tmp_path / "w.bin"), (nz, ny, nx)), vec[:3])
    # 2D: [x][y](, k) in the file
    s2 = scal[0]
    s2.T.astype(np.float64).tofile(tmp_path / "s2.bin")
    np.testing.assert_array_equal(cio.import_scalar_field_from_chfem(str(tmp_path / "s2.bin"), (ny, nx)), s2)
    v2 = np.stack([s2, s2 + 1000])
    v2.transpose(2, 1, 0).astype(np.float64).tofile(tmp_path / "v2.bin")
    np.testing.assert_array_equal(cio.import_vector_field_from_chfem(str(tmp_path / "v2.bin"), (ny, nx)), v2)


def test_output_fields_directory_checked():
    from chfem_b200 import compute_property
    img = np.zeros((4, 4, 4), np.uint8)
    with pytest.raises(ValueError, match="does not exist"):
        compute_property("conductivity", img, {0: 1.0}, output_fields="/nonexistent_dir_xyz/cube")
    with pytest.raises(ValueError, match="Two-vectors solvers"):
        compute_property("conductivity", img, {0: 1.0}, solver="cg2", output_fields="cube")


# ---- GPU: chfem_b200's fields -------------------------------------------------------------
FIELD_CASES = [
    ("gth3", 0, (6, 7, 5), 3, 1, []),
    ("gth2_ebe", 0, (5, 6, 7), 2, 1, ["-p", "1"]),
    ("gel3", 1, (6, 5, 7), 3, 1, []),
    ("gel2_ref2", 1, (3, 4, 3), 2, 2, []),
]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["single", "block"])
@pytest.mark.parametrize("name,analysis,shape,nmat,refinement,flags", FIELD_CASES)
def test_gpu_fields(tmp_path, name, analysis, shape, nmat, refinement, flags, mode):
    img, nf, raw = _case(tmp_path, name, analysis, shape, nmat, refinement)
    prefix = nf[:-3]
    H.run_exec(H.ORACLE_EXEC, nf, raw, "-e", *flags, env=ONE_THREAD)
    sol, fld, _, _ = CASE_FILES[analysis]
    ref = {f: np.fromfile(f) for f in glob.glob(prefix + "_*.bin")}
    for f in ref:
        os.remove(f)
    extra = ["--multirhs"] if mode == "block" else []
    H.run_exec(H.CHFEM_EXEC, nf, raw, "-e", *flags, *extra)
    ours = {f: np.fromfile(f) for f in glob.glob(prefix + "_*.bin")}
    assert sorted(ours) == sorted(ref)
    # the device field kernel on our own solution: same arithmetic as the oracle
    _check_fields_against_oracle(prefix, img, nf, analysis, refinement, 1e-11)
    # solution and field against the reference's (tolerance 1e-10 solves)
    for f in ref:
        assert ours[f].shape == ref[f].shape
        assert H.rel_to_max(ours[f], ref[f]) < 1e-6, (f, H.rel_to_max(ours[f], ref[f]))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["single", "block"])
def test_gpu_stokes_fields(tmp_path, mode):
    from chfem_b200.synthetic import pore_grf
    img = pore_grf((10, 12, 14), corr=2.0, porosity=0.5, seed=11)
    nf, raw = H.write_small_case(str(tmp_path), "fst", img, 2, tol=1e-10, maxit=20000, solver=1)
    prefix = nf[:-3]
    H.run_exec(H.ORACLE_EXEC, nf, raw, "-e", env=ONE_THREAD)
    ref = {f: np.fromfile(f) for f in glob.glob(prefix + "_*.bin")}
    for f in ref:
        os.remove(f)
    assert len(ref) == 6
    H.run_exec(H.CHFEM_EXEC, nf, raw, "-e", *(["--multirhs"] if mode == "block" else []))
    ours = {f: np.fromfile(f) for f in glob.glob(prefix + "_*.bin")}
    assert sorted(ours) == sorted(ref)
    for f in ref:
        assert ours[f].shape == ref[f].shape
        assert H.rel_to_max(ours[f], ref[f]) < 1e-6, (f, H.rel_to_max(ours[f], ref[f]))
        if "velocity" in f:  # solid nodes carry no velocity
            solid = (img == 255).transpose(0, 2, 1).reshape(-1)
            u = ours[f].reshape(-1, 3)
            assert np.all(u[solid] == 0.0)


@pytest.mark.gpu
def test_gpu_compute_property_output_fields(tmp_path):
    from chfem_b200 import compute_property
    img = H.small_image((6, 8, 10), 2, seed=3)
    prefix = str(tmp_path / "cube")
    C = compute_property("elasticity", img, {0: (1.0, 0.3), 255: (10.0, 0.2)}, direction="x", output_fields=prefix,
                         solver_tolerance=1e-10)
    assert np.isfinite(C).all()
    assert not os.path.exists(prefix + ".nf")
    u = cio.import_vector_field_from_chfem(prefix + "_displacement_0.bin", img.shape)
    s = cio.import_stress_field_from_chfem(prefix + "_stress_0.bin", img.shape)
    assert u.shape == (3,) + img.shape and s.shape == (6,) + img.shape
    # the mean of sigma_xx over the nodes is C[0][0] of the x load case (unit macroscopic strain)
    assert abs(s[0].mean() - C[0][0]) < 1e-6 * abs(C[0][0])
    assert not os.path.exists(prefix + "_displacement_1.bin")
    # no fields without the request
    C2 = compute_property("elasticity", img, {0: (1.0, 0.3), 255: (10.0, 0.2)}, direction="y", solver_tolerance=1e-10)
    assert not os.path.exists(prefix + "_displacement_1.bin")
