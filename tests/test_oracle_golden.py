"""The oracle (reference host code + CPU restatement of its solver) reproduces the reference's
own golden effective tensors (test/input/3D/*_result.bin, test/input/2D/*_result.bin) within the reference's
regression tolerance of 1e-4 relative to the largest entry (test/test_chfem.c:5,340-351)."""
import os

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.skipif(not H.oracle_available(), reason="oracle/_ref not built (needs the reference tree)")


@pytest.mark.parametrize("name", ["thermal_ggg40", "fluid_fibers", "elastic_ggg40"])
def test_oracle_matches_golden(tmp_path, name):
    nf, raw, meta = H.golden_case_files(name, str(tmp_path))
    C, out = H.run_exec(H.ORACLE_EXEC, nf, raw, "-d", meta["direction"], env={"OMP_NUM_THREADS": str(os.cpu_count() or 4)})
    col = C[:, meta["direction"]]
    assert H.rel_to_max(col, meta["column"]) < meta["reference_tolerance"]


@pytest.mark.parametrize("name,par", [("thermal_2d", "0"), ("thermal_2d", "1"), ("elastic_2d", "0"), ("elastic_2d", "1"),
                                      ("fluid_2d", "0")])
def test_oracle_matches_golden_2d(tmp_path, name, par):
    """2D pixel models (test/input/2D): every load case, node-by-node and (thermal, elastic)
    element-by-element."""
    nf, raw, meta = H.golden_case_files(name, str(tmp_path))
    C, out = H.run_exec(H.ORACLE_EXEC, nf, raw, "-p", par, env={"OMP_NUM_THREADS": str(os.cpu_count() or 4)})
    assert H.rel_to_max(C, meta["tensor"]) < meta["reference_tolerance"]


def test_oracle_standalone_builds():
    path = os.path.join(H.ROOT, "oracle", "liboracle_cudapcg.so")
    assert os.path.exists(path)
    import ctypes
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    assert lib.cudapcgInit(1, 0) == 1 and lib.cudapcgEnd() == 1
