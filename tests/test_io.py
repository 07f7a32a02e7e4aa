"""chfem .nf / .raw formats (chfem/io.py) and the compute_property argument checks."""
import numpy as np
import pytest

from chfem_b200 import compute_property, export_for_chfem, import_nf, import_raw
from tests import helpers as H


def test_nf_roundtrip(tmp_path):
    img = H.small_image((4, 5, 6), 2, seed=1)
    d = export_for_chfem(str(tmp_path / "a.raw"), img, 1, mat_props={0: (1.0, 0.3), 255: (10.0, 0.2)}, voxel_size=2.0,
                         solver_tolerance=1e-5, solver_maxiter=77)
    nf = import_nf(str(tmp_path / "a.nf"))
    assert nf["image_dimensions"] == (4, 5, 6)
    assert nf["type_of_analysis"] == 1 and nf["number_of_iterations"] == 77
    assert nf["properties_of_materials"] == [(0, 1.0, 0.3), (255, 10.0, 0.2)]
    assert abs(nf["solver_tolerance"] - 1e-5) < 1e-20 and nf["voxel_size"] == 2.0
    back = import_raw(str(tmp_path / "a.raw"), (4, 5, 6))
    assert np.array_equal(back, img)
    assert d["image_dimensions"] == [6, 5, 4]


def test_golden_nf_parses():
    g = H.golden()
    nf = import_nf(H.GOLDEN + "/" + g["fluid_fibers"]["nf"])
    assert nf["refinement"] == 2 and nf["image_dimensions"] == (10, 100, 100)


def test_compute_property_argument_errors():
    a = np.zeros((4, 4, 4), np.uint8)
    with pytest.raises(ValueError, match="Invalid property"):
        compute_property("viscosity", a)
    with pytest.raises(ValueError, match="Invalid direction"):
        compute_property("conductivity", a, mat_props={0: 1.0}, direction="w")
    with pytest.raises(ValueError, match="Invalid solver"):
        compute_property("conductivity", a, mat_props={0: 1.0}, solver="gmres")
    with pytest.raises(ValueError, match="uint8"):
        compute_property("conductivity", a.astype(np.int32), mat_props={0: 1.0})
    with pytest.raises(ValueError, match="No fluid phase"):
        compute_property("conductivity", a + 3, mat_props={3: 1.0})
    with pytest.raises(ValueError, match="Material properties"):
        compute_property("conductivity", a)
