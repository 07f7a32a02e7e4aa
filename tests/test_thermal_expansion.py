"""Effective thermal expansion (elasticity with a thermal expansion coefficient per material:
the .nf %thermal_expansion list, compute_property mat_props {phase: (E, nu, alpha)}).

The reference runs one more solve after the six load cases, under a unit temperature rise
(femhmg.c:1121-1168, femhmg_elastic_3D.c:464-505 and :863-1074), and writes the six effective
coefficients after the tensor (femhmg.c:1359-1364).  CPU: the oracle (the reference's own host
code) on a homogeneous image returns the material's coefficient.  GPU: chfem_b200 against the
oracle, one-by-one and block solves, FP64 and mixed, and through compute_property.
"""
import os
import subprocess
import tempfile
import zlib

import numpy as np
import pytest

from tests import helpers as H

needs_oracle = pytest.mark.skipif(not H.oracle_available(), reason="oracle executable not built")


def write_case(workdir, name, img, props, tol=1e-10):
    from chfem_b200.io import export_for_chfem
    prefix = os.path.join(str(workdir), name)
    export_for_chfem(prefix + ".raw", img, 1, mat_props=props, solver_tolerance=tol, solver_maxiter=20000)
    return prefix + ".nf", prefix + ".raw"


def run_tensor_and_alpha(exe, nf, raw, *flags, env=None, dim=3):
    """The tensor and the expansion from the -b file: 36 + 6 values in 3D, 9 + 3 in 2D."""
    out = tempfile.mktemp(suffix=".bin")
    p = subprocess.run([exe, nf, raw, "-b", out, *flags], capture_output=True, text=True, timeout=1800,
                       env=None if env is None else {**os.environ, **env})
    assert p.returncode == 0 and os.path.exists(out), p.stdout[-2000:] + p.stderr[-2000:]
    v = np.fromfile(out)
    os.remove(out)
    n = 6 if dim == 3 else 3
    assert v.size == n * n + n, v.size
    return v[:n * n].reshape(n, n), v[n * n:], p.stdout


@needs_oracle
def test_oracle_homogeneous_expansion(tmp_path):
    img = np.full((4, 5, 6), 255, np.uint8)
    img[0, 0, 0] = 0  # a second colour listed with the same properties
    props = {0: (3.0, 0.25, 1.5e-5), 255: (3.0, 0.25, 1.5e-5)}
    nf, raw = write_case(tmp_path, "hom", img, props)
    C, a, _ = run_tensor_and_alpha(H.ORACLE_EXEC, nf, raw)
    np.testing.assert_allclose(a, [1.5e-5, 1.5e-5, 1.5e-5, 0, 0, 0], atol=1e-12)


@needs_oracle
def test_oracle_homogeneous_expansion_2d(tmp_path):
    """2D (femhmg_elastic_2D.c:277-300, :388-528): the in-plane expansion (xx, yy, xy) of a
    homogeneous image is the material's, in the reference's default plane-strain build."""
    img = np.full((5, 7), 255, np.uint8)
    img[0, 0] = 0
    props = {0: (3.0, 0.25, 1.5e-5), 255: (3.0, 0.25, 1.5e-5)}
    nf, raw = write_case(tmp_path, "hom2", img, props)
    C, a, log = run_tensor_and_alpha(H.ORACLE_EXEC, nf, raw, dim=2)
    np.testing.assert_allclose(a, [1.5e-5, 1.5e-5, 0], atol=1e-12)


CASES = [("te2", (6, 7, 8), 2, {0: (1.0, 0.3, 2e-5), 255: (10.0, 0.2, 1e-5)}),
         ("te2b", (8, 6, 7), 2, {0: (1.0, 0.3, 3e-5), 255: (4.0, 0.25, -5e-6)})]


@pytest.mark.gpu
def test_gpu_three_materials_scan_limit(tmp_path):
    """With three materials the %thermal_expansion entry of a written .nf lies past the
    reference's 12-entry scan (femhmg.c:1456-1586): neither program reads it, both return the
    tensor alone."""
    img = H.small_image((6, 6, 6), 3, seed=9)
    props = {0: (1.0, 0.3, 3e-5), 255: (10.0, 0.2, 1e-5), 100: (4.0, 0.25, -5e-6)}
    nf, raw = write_case(tmp_path, "te3", img, props)
    sizes = []
    for exe in (H.ORACLE_EXEC, H.CHFEM_EXEC):
        out = str(tmp_path / "o.bin")
        p = subprocess.run([exe, nf, raw, "-b", out], capture_output=True, text=True, timeout=1800)
        assert p.returncode == 0
        sizes.append(np.fromfile(out).size)
    assert sizes == [36, 36]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [[], ["--multirhs"], ["--precision", "mixed"], ["--multirhs", "--precision", "mixed"]])
@pytest.mark.parametrize("name,shape,nmat,props", CASES)
def test_gpu_thermal_expansion_vs_oracle(tmp_path, name, shape, nmat, props, mode):
    img = H.small_image(shape, nmat, seed=zlib.crc32(name.encode()) % 10000)
    nf, raw = write_case(tmp_path, name, img, props)
    Cref, aref, _ = run_tensor_and_alpha(H.ORACLE_EXEC, nf, raw)
    C, a, log = run_tensor_and_alpha(H.CHFEM_EXEC, nf, raw, *mode)
    assert "Effective thermal expansion" in log
    tol = 1e-6 if "mixed" not in mode else 1e-4
    assert H.rel_to_max(C, Cref) < tol
    assert H.rel_to_max(a, aref) < tol, (a, aref)


@pytest.mark.gpu
def test_gpu_compute_property_thermal_expansion(tmp_path):
    from chfem_b200 import compute_property
    name, shape, nmat, props = CASES[0]
    img = H.small_image(shape, nmat, seed=zlib.crc32(name.encode()) % 10000)
    nf, raw = write_case(tmp_path, name, img, props)
    Cref, aref, _ = run_tensor_and_alpha(H.ORACLE_EXEC, nf, raw)
    out = compute_property("elasticity", img, props, solver_tolerance=1e-10, solver_maxiter=20000)
    assert len(out) == 7 and len(out[6]) == 6
    assert H.rel_to_max(np.array(out[:6]), Cref) < 1e-6
    assert H.rel_to_max(np.array(out[6]), aref) < 1e-6
    with pytest.raises(ValueError, match="Must be"):
        compute_property("elasticity", img, props, direction="x")


CASES_2D = [("te2d", (17, 23), {0: (1.0, 0.3, 2e-5), 255: (10.0, 0.2, 1e-5)}),
            ("te2d_neg", (21, 14), {0: (1.0, 0.3, 3e-5), 255: (4.0, 0.25, -5e-6)})]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [[], ["--precision", "mixed"]])
@pytest.mark.parametrize("name,shape,props", CASES_2D)
def test_gpu_thermal_expansion_2d_vs_oracle(tmp_path, name, shape, props, mode):
    """2D images: the tensor and the in-plane expansion (xx, yy, xy) against the oracle (the
    reference's host code, plane strain), and the 2 x 2 expansion printout."""
    img = H.small_image(shape, 2, seed=zlib.crc32(name.encode()) % 10000)
    nf, raw = write_case(tmp_path, name, img, props)
    Cref, aref, _ = run_tensor_and_alpha(H.ORACLE_EXEC, nf, raw, dim=2)
    C, a, log = run_tensor_and_alpha(H.CHFEM_EXEC, nf, raw, *mode, dim=2)
    assert "Effective thermal expansion" in log
    tol = 1e-6 if "mixed" not in mode else 1e-4
    assert H.rel_to_max(C, Cref) < tol
    assert H.rel_to_max(a, aref) < tol, (a, aref)


@pytest.mark.gpu
def test_gpu_thermal_expansion_2d_plane_stress_homogeneous(tmp_path):
    """Plane stress (CHFEM_B200_PLANE_STRESS=1): the load and the stresses take the element
    matrices' plane-stress matrix, so a homogeneous image returns its own expansion and the
    tensor E / (1 - nu^2) [1 nu 0; nu 1 0; 0 0 (1 - nu) / 2]."""
    img = np.full((9, 11), 255, np.uint8)
    img[2, 3] = 0
    E, nu, al = 3.0, 0.25, 1.5e-5
    props = {0: (E, nu, al), 255: (E, nu, al)}
    nf, raw = write_case(tmp_path, "hps", img, props)
    C, a, _ = run_tensor_and_alpha(H.CHFEM_EXEC, nf, raw, env={"CHFEM_B200_PLANE_STRESS": "1"}, dim=2)
    f = E / (1 - nu * nu)
    np.testing.assert_allclose(C, f * np.array([[1, nu, 0], [nu, 1, 0], [0, 0, 0.5 * (1 - nu)]]), atol=1e-8 * f)
    np.testing.assert_allclose(a, [al, al, 0], atol=1e-12)


@pytest.mark.gpu
def test_gpu_compute_property_thermal_expansion_2d(tmp_path):
    from chfem_b200 import compute_property
    name, shape, props = CASES_2D[0]
    img = H.small_image(shape, 2, seed=zlib.crc32(name.encode()) % 10000)
    nf, raw = write_case(tmp_path, name, img, props)
    Cref, aref, _ = run_tensor_and_alpha(H.ORACLE_EXEC, nf, raw, dim=2)
    out = compute_property("elasticity", img, props, solver_tolerance=1e-10, solver_maxiter=20000)
    assert len(out) == 4 and len(out[3]) == 3
    assert H.rel_to_max(np.array(out[:3]), Cref) < 1e-6
    assert H.rel_to_max(np.array(out[3]), aref) < 1e-6
