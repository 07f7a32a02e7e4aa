"""Batched thermal homogenization (compute_conductivity_batch / cudapcgB200SolveThermalBatch)
against the one-image-at-a-time path on the GPU.

Bars: FP64 tensors within 1e-6 of compute_property's relative to the largest entry (the same
recurrence and stopping test per load case; iteration counts within +-1, the summation order of
the operator differs), mixed precision within 1e-4; a one-phase image gives k I; two runs are
bitwise identical (deterministic reductions).
"""
import zlib

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu

SIZES = [(8, 9, 10), (12, 12, 12), (16, 8, 20), (5, 7, 9), (20, 20, 4), (3, 33, 6), (1, 9, 17)]


def batch_images(sizes, seed0=0, three_phase=()):
    imgs, props = [], []
    for i, shp in enumerate(sizes):
        rng = np.random.default_rng(seed0 + i)
        if i in three_phase:
            img = rng.choice(np.array([0, 100, 255], np.uint8), size=shp)
            props.append({0: 1.0, 100: float(rng.uniform(2, 5)), 255: float(rng.uniform(5, 50))})
        else:
            img = H.small_image(shp, 2, seed=zlib.crc32(f"b{seed0}{i}".encode()) % 10000)
            props.append({0: 1.0, 255: float(np.exp(rng.uniform(np.log(2), np.log(100))))})
        imgs.append(img)
    return imgs, props


def single(img, props, precision="fp64"):
    from chfem_b200 import compute_property, _native
    C = np.array(compute_property("conductivity", img, mat_props=props, solver_tolerance=1e-8, solver_maxiter=20000,
                                  precision=precision))
    st = _native.solve_stats()
    return C, [st.iterations[k] for k in range(3)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_single(precision):
    from chfem_b200 import compute_conductivity_batch
    imgs, props = batch_images(SIZES, three_phase=(2,))
    Cb, its = compute_conductivity_batch(imgs, props, solver_tolerance=1e-8, solver_maxiter=20000, precision=precision,
                                         return_iterations=True)
    for i, (img, p) in enumerate(zip(imgs, props)):
        C1, its1 = single(img, p)
        tol = 1e-6 if precision == "fp64" else 1e-4
        assert H.rel_to_max(Cb[i], C1) < tol, (i, Cb[i], C1)
        if precision == "fp64":
            assert all(abs(int(a) - int(b)) <= 1 for a, b in zip(its[i], its1)), (i, its[i], its1)
        else:
            assert all(int(a) <= 2 * int(b) + 50 for a, b in zip(its[i], its1)), (i, its[i], its1)


def test_batch_homogeneous_and_deterministic():
    from chfem_b200 import compute_conductivity_batch
    imgs, props = batch_images(SIZES[:4], seed0=7)
    imgs.append(np.zeros((10, 6, 8), np.uint8))
    props.append({0: 3.5})
    C1 = compute_conductivity_batch(imgs, props, solver_tolerance=1e-10)
    C2 = compute_conductivity_batch(imgs, props, solver_tolerance=1e-10)
    assert np.array_equal(C1, C2)
    assert np.allclose(C1[-1], 3.5 * np.eye(3), atol=1e-9)


def test_batch_many_uneven_samples():
    """Enough samples of uneven sizes that CTA slices cross many sample boundaries."""
    from chfem_b200 import compute_conductivity_batch
    rng = np.random.default_rng(11)
    sizes = [tuple(int(v) for v in rng.choice([4, 8, 12, 16, 24], size=3)) for _ in range(60)]
    imgs, props = batch_images(sizes, seed0=100)
    Cb = compute_conductivity_batch(imgs, props, solver_tolerance=1e-8, solver_maxiter=20000)
    for i in range(0, 60, 7):
        C1, _ = single(imgs[i], props[i])
        assert H.rel_to_max(Cb[i], C1) < 1e-6, (i, sizes[i])
    # a larger batch member against the oracle CLI
    i = int(np.argmax([np.prod(s) for s in sizes]))
    import tempfile, os
    d = tempfile.mkdtemp()
    from chfem_b200.io import export_for_chfem
    export_for_chfem(os.path.join(d, "o.raw"), imgs[i], 0, mat_props=props[i], solver_tolerance=1e-8, solver_maxiter=20000)
    Cref, _ = H.run_exec(H.ORACLE_EXEC, os.path.join(d, "o.nf"), os.path.join(d, "o.raw"))
    assert H.rel_to_max(Cb[i], Cref) < 1e-6
