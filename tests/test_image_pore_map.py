"""Image pore map (-pm 0, CUDAPCG_POREMAP_IMG; femhmg.c:476-513, :962-965, cudapcg.cu:336-363).

With -pm 0 the host hands the solver every node's fluid key and the node->DOF map instead of
the DOF->node map and the interface keys; the unknowns, their numbering and the operator are
the same.  CPU: the oracle (the reference's host code in its image-map mode, with the DOF->node
map and the interface keys scattered from the two maps it receives) gives the -pm 1 tensor.
GPU: chfem_b200 with -pm 0 equals the oracle with -pm 0, and its own -pm 1 result, for 3D and
2D Stokes, MINRES and CG, the block solve and the 2-vector solver.
"""
import zlib

import numpy as np
import pytest

from tests import helpers as H

needs_oracle = pytest.mark.skipif(not H.oracle_available(), reason="oracle executable not built")


def _case(tmp_path, name, shape, porosity, solver=1):
    rng = np.random.default_rng(zlib.crc32(name.encode()) % 10000)
    img = np.where(rng.random(shape) < porosity, 0, 255).astype(np.uint8)
    return H.write_small_case(str(tmp_path), name, img, 2, tol=1e-9, maxit=20000, solver=solver)


@needs_oracle
@pytest.mark.parametrize("name,shape", [("pm3", (8, 9, 10)), ("pm2", (21, 17))])
def test_oracle_image_pore_map(tmp_path, name, shape):
    nf, raw = _case(tmp_path, name, shape, 0.6)
    Cnum, lognum = H.run_exec(H.ORACLE_EXEC, nf, raw, "-pm", "1")
    Cimg, logimg = H.run_exec(H.ORACLE_EXEC, nf, raw, "-pm", "0")
    assert H.rel_to_max(Cimg, Cnum) < 1e-9
    assert H.parse_iterations(logimg) == H.parse_iterations(lognum)


@pytest.mark.gpu
@needs_oracle
@pytest.mark.parametrize("name,shape,flags", [("g3_minres", (12, 13, 14), []), ("g3_cg", (10, 11, 9), ["-s", "0"]),
                                              ("g2_minres", (25, 22), []), ("g3_block", (12, 10, 11), ["--multirhs"])])
def test_image_pore_map_vs_oracle(tmp_path, name, shape, flags):
    nf, raw = _case(tmp_path, name, shape, 0.55)
    Cref, _ = H.run_exec(H.ORACLE_EXEC, nf, raw, "-pm", "0", *[f for f in flags if f != "--multirhs"])
    C0, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-pm", "0", *flags)
    C1, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-pm", "1", *flags)
    assert H.rel_to_max(C0, Cref) < 1e-6
    assert H.rel_to_max(C0, C1) < 1e-12


@pytest.mark.gpu
def test_image_pore_map_two_vector(tmp_path):
    """PMINRES2 (-s 5) under the image map: the reduced velocities, hence the tensor, equal the
    DOF-number map's (the reference leaves its 2-vector kernels unimplemented for this map,
    wrappers.cu:653-665)."""
    nf, raw = _case(tmp_path, "tv", (12, 12, 12), 0.6)
    C0, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-pm", "0", "-s", "5")
    C1, _ = H.run_exec(H.CHFEM_EXEC, nf, raw, "-pm", "1", "-s", "5")
    assert H.rel_to_max(C0, C1) < 1e-12
