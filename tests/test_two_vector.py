"""The 2-vector Stokes solvers (CG2 / PCG2 / MINRES2 / PMINRES2) with on-the-fly reduction of
the solution (chfem_exec -s 4 / -s 5, -u 0/1/2).

CPU: the oracle's restatement of these solvers is pinned on the reference's own CUDA build
(tests/golden/two_vector_ref.json for 3D images and two_vector_2d_ref.json for 2D images, made
by tests/golden/make_two_vector_fixture.py): tensors, iteration counts and the per-step
reductions it writes to <nf>_xreduce_metrics_<n>.bin.
GPU: the B200 library against the oracle on the same runs, its device memory, and the Python
entry point.
"""
import ctypes
import json
import os
import shutil

import numpy as np
import pytest

from tests import helpers as H

FIXTURE = os.path.join(H.GOLDEN, "two_vector_ref.json")
FIXTURE_2D = os.path.join(H.GOLDEN, "two_vector_2d_ref.json")
needs_oracle = pytest.mark.skipif(not H.oracle_available(), reason="oracle executable not built")


def fixture(path=FIXTURE):
    with open(path) as f:
        return json.load(f)


def _image(spec):
    """The generator's images: a percolating GRF pore space (3D), seeded uniform pixels (2D)."""
    if len(spec["shape"]) == 2:
        rng = np.random.default_rng(spec["seed"])
        return np.where(rng.random(tuple(spec["shape"])) < spec["porosity"], 0, 255).astype(np.uint8)
    from chfem_b200.synthetic import pore_grf
    return pore_grf(tuple(spec["shape"]), corr=spec["corr"], porosity=spec["porosity"], seed=spec["seed"])


def make_case(workdir, name, spec, maxit=20000, suffix=""):
    from chfem_b200.io import export_for_chfem
    img = _image(spec)
    prefix = os.path.join(str(workdir), name + suffix)
    export_for_chfem(prefix + ".raw", img, 2, mat_props=None, voxel_size=spec["voxel"], solver_type=1, refinement=1,
                     export_raw=True, export_nf=True, solver_tolerance=spec["tol"], solver_maxiter=maxit)
    return prefix + ".nf", prefix + ".raw"


def read_metrics(prefix, ncases=3):
    return [np.fromfile(f"{prefix}_xreduce_metrics_{k}.bin") for k in range(1, ncases + 1)]


def clear_metrics(workdir):
    for f in os.listdir(workdir):
        if "_xreduce_metrics_" in f:
            os.remove(os.path.join(workdir, f))


def iterations_close(its, ref, flags, dim=3):
    """Same counts (+-1) with Jacobi and the residual norms.  The error norm is a step-size test
    and the unpreconditioned recurrences amplify rounding, so there the summation order (the
    reference's GPU reductions, the oracle's threaded sums, the B200 passes) moves the stop by
    a few steps.  On the 2D pixel images the stopping step is dominated by rounding: the
    reference's own MINRES and MINRES2 stop 7 steps apart on pix22x35_h05, and the oracle's
    counts there move between 141 and 160 from run to run (its threaded sums combine in
    run-dependent order, and the B200's MINRES2 with the error norm stopped at 163 where the
    oracle stopped at 147); MINRES-family counts are held to 15 %, CG-family ones not at all."""
    assert len(its) == len(ref)
    if dim == 2:
        if flags[flags.index("-s") + 1] in ("0", "4"):
            return
        for a, b in zip(its, ref):
            assert abs(a - b) <= max(2, int(0.15 * b)) + (max(3, int(0.03 * b)) if "-j" in flags else 0), (its, ref)
        return
    slack = 1
    if "-c" in flags and flags[flags.index("-c") + 1] == "2":
        slack = 3
    for a, b in zip(its, ref):
        tol = max(3, int(0.03 * b)) if "-j" in flags else slack
        assert abs(a - b) <= tol, (its, ref)


def run_with_guess(exe, tmp_path, name, spec, nf, raw, flags):
    """-xi with a 20-step MINRES solution of the same model as the guess."""
    nf20, _ = make_case(tmp_path, name, spec, maxit=20, suffix="_guess")
    H.run_exec(exe, nf20, raw, "-s", "1", "-xo")
    return H.run_exec(exe, nf, raw, *flags[:-1], nf20[:-3] + "_X")


# ---- CPU: the oracle on the reference's own runs ----------------------------------------
def _fixture_runs():
    out = []
    for path in (FIXTURE, FIXTURE_2D):
        if os.path.exists(path):
            out += [(os.path.basename(path), name, i) for name, case in fixture(path)["cases"].items() for i in range(len(case["runs"]))]
    return out


@needs_oracle
@pytest.mark.parametrize("fname,name,i", _fixture_runs())
def test_oracle_matches_reference_two_vector_runs(tmp_path, fname, name, i):
    case = fixture(os.path.join(H.GOLDEN, fname))["cases"][name]
    spec, run = case["spec"], case["runs"][i]
    ncases = len(spec["shape"])  # load cases: 3 on a 3D image, 2 on a 2D one
    flags = run["flags"]
    if flags == ["-s", "4", "-c", "2"] and ncases == 3:
        pytest.skip("reference defect: see test_reference_pcg2_error_norm_defect")
    if ncases == 2 and flags[:2] == ["-s", "4"] and not ("-u" in flags and flags[flags.index("-u") + 1] != "2"):
        cg = {tuple(r["flags"]): r for r in case["runs"]}[("-s", "0")]
        if H.rel_to_max(run["C"], cg["C"]) > 1e-7:
            pytest.skip("reference defect: its PCG2 FULL-mode tensor departs from its own PCG tensor "
                        "(test_reference_pcg2_2d_full_defect)")
    nf, raw = make_case(tmp_path, name, spec)
    if "-xi" in flags:
        C, log = run_with_guess(H.ORACLE_EXEC, tmp_path, name, spec, nf, raw, flags)
    else:
        C, log = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags)
    assert H.rel_to_max(C, np.array(run["C"])) < 1e-7, (flags, H.rel_to_max(C, np.array(run["C"])))
    its = H.parse_iterations(log)
    iterations_close(its, run["iterations"], flags, ncases)
    if "metrics" in run:
        full = "-u" not in flags or flags[flags.index("-u") + 1] == "2"
        ncomp = 1 if ("-u" in flags and flags[flags.index("-u") + 1] == "1") else ncases
        for k, (got, ref) in enumerate(zip(read_metrics(nf[:-3], ncases), run["metrics"])):
            ref = np.asarray(ref)
            if its[k] != run["iterations"][k]:
                continue  # a step more or less (threaded sums): the tensor column is checked above
            assert got.size == ref.size
            if full:
                # The reference's FULL-mode sums of the accumulator read past the partials its
                # strided reduction wrote, so its intermediate entries carry leftovers of the
                # previous reduction (which vanish as the iteration converges); its last entries,
                # the tensor column, are exact.  NONE and ONLYDIR entries are exact throughout.
                g, r = got.reshape(ncomp, -1), ref.reshape(ncomp, -1)
                assert np.abs(g[:, -1] - r[:, -1]).max() < 1e-7 * np.abs(r[:, -1]).max()
            else:
                assert H.rel_to_max(got, ref) < 1e-7


def test_reference_pcg2_error_norm_defect():
    """The reference's PCG2 with the error norm (-s 4 -c 2) stops at the same iteration as with
    the L2 norm but reports a tensor several percent away from its own converged one: its
    FULL-mode sums of the accumulator pick up leftovers of the reduction run just before them,
    which for this norm is max|x| and does not vanish at convergence.  chfem_b200 and the oracle
    return the converged tensor there; this records the reference's behaviour."""
    for name, case in fixture()["cases"].items():
        runs = {tuple(r["flags"]): r for r in case["runs"]}
        bad, good = runs[("-s", "4", "-c", "2")], runs[("-s", "4")]
        assert bad["iterations"] == good["iterations"]
        assert H.rel_to_max(bad["C"], good["C"]) > 1e-3


def test_fixture_two_vector_equals_full_solvers():
    """In the reference, CG2 / MINRES2 reproduce CG / MINRES's tensor (the reduced sums are the
    velocity averages the full solvers' tensor update forms), on 3D and 2D images (2D: PCG2
    without an accumulator, -u 0, and MINRES2; see test_reference_pcg2_2d_full_defect)."""
    for name, case in fixture()["cases"].items():
        runs = {tuple(r["flags"]): r for r in case["runs"]}
        assert H.rel_to_max(runs[("-s", "5")]["C"], runs[("-s", "1")]["C"]) < 1e-7
        assert H.rel_to_max(runs[("-s", "4")]["C"], runs[("-s", "0")]["C"]) < 1e-7
        assert runs[("-s", "5")]["iterations"] == runs[("-s", "1")]["iterations"]
    for name, case in fixture(FIXTURE_2D)["cases"].items():
        runs = {tuple(r["flags"]): r for r in case["runs"]}
        assert H.rel_to_max(runs[("-s", "5")]["C"], runs[("-s", "1")]["C"]) < 1e-7
        assert H.rel_to_max(runs[("-s", "4", "-u", "0")]["C"], runs[("-s", "0")]["C"]) < 1e-7


def test_reference_pcg2_2d_full_defect():
    """On the 2D image pix30x26 the reference's PCG2 with the accumulator (FULL, -u 2: the
    default and -c 2) stops where its PCG does but returns a tensor 1.9e-5 away from it, while
    its PCG2 without an accumulator (-u 0) agrees to 1e-10: the FULL-mode sums pick up leftovers
    of an earlier reduction (as in test_reference_pcg2_error_norm_defect).  chfem_b200 and the
    oracle return the PCG tensor there; this records the reference's behaviour."""
    runs = {tuple(r["flags"]): r for r in fixture(FIXTURE_2D)["cases"]["pix30x26"]["runs"]}
    for bad in (("-s", "4"), ("-s", "4", "-c", "2")):
        assert runs[bad]["iterations"] == runs[("-s", "0")]["iterations"]
        assert H.rel_to_max(runs[bad]["C"], runs[("-s", "0")]["C"]) > 1e-6
    assert H.rel_to_max(runs[("-s", "4", "-u", "0")]["C"], runs[("-s", "0")]["C"]) < 1e-9


# ---- GPU: the B200 library ---------------------------------------------------------------
GPU_FLAGS = [["-s", "5"], ["-s", "5", "-u", "0"], ["-s", "5", "-u", "1"], ["-s", "5", "-j", "0"], ["-s", "5", "-c", "1"],
             ["-s", "5", "-c", "2"], ["-s", "4"], ["-s", "4", "-u", "0"], ["-s", "4", "-u", "1"], ["-s", "4", "-j", "0"],
             ["-s", "4", "-c", "1"], ["-s", "4", "-c", "2"], ["-s", "4", "-c", "2", "-u", "0"]]


@pytest.mark.gpu
@pytest.mark.parametrize("fname,name", [("two_vector_ref.json", "pore16"), ("two_vector_ref.json", "pore12_h05"),
                                        ("two_vector_2d_ref.json", "pix30x26"), ("two_vector_2d_ref.json", "pix22x35_h05")])
@pytest.mark.parametrize("flags", GPU_FLAGS)
def test_gpu_two_vector_vs_oracle(tmp_path, fname, name, flags):
    spec = fixture(os.path.join(H.GOLDEN, fname))["cases"][name]["spec"]
    ncases = len(spec["shape"])
    nf, raw = make_case(tmp_path, name, spec)
    Cref, logref = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags)
    mref = read_metrics(nf[:-3], ncases)
    clear_metrics(str(tmp_path))
    C, log = H.run_exec(H.CHFEM_EXEC, nf, raw, *flags)
    assert "Effective fields" in log
    assert H.rel_to_max(C, Cref) < 1e-7, H.rel_to_max(C, Cref)
    its, itsref = H.parse_iterations(log), H.parse_iterations(logref)
    iterations_close(its, itsref, flags, ncases)
    m = read_metrics(nf[:-3], ncases)
    for k in range(ncases):
        n = its[k] + 1
        assert m[k].size % n == 0
        if its[k] == itsref[k] and "-j" not in flags:
            # per-step sums of the iterates
            assert m[k].size == mref[k].size
            assert H.rel_to_max(m[k], mref[k]) < 1e-6
        elif its[k] == itsref[k]:
            # without Jacobi, rounding grows along the recurrence on the indefinite Stokes system:
            # the iterates drift apart at 1e-3 while the last sums (the tensor column) agree
            g, r = m[k].reshape(-1, n), mref[k].reshape(-1, n)
            assert np.abs(g[:, -1] - r[:, -1]).max() < 1e-7 * np.abs(r[:, -1]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [["-s", "5", "-xi"], ["-s", "4", "-xi"]])
def test_gpu_two_vector_initial_guess(tmp_path, flags):
    spec = fixture()["cases"]["pore16"]["spec"]
    nf, raw = make_case(tmp_path, "pore16", spec)
    Cref, logref = run_with_guess(H.ORACLE_EXEC, tmp_path, "pore16", spec, nf, raw, flags + ["x"])
    C, log = run_with_guess(H.CHFEM_EXEC, tmp_path, "pore16", spec, nf, raw, flags + ["x"])
    assert H.rel_to_max(C, Cref) < 1e-7
    iterations_close(H.parse_iterations(log)[-3:], H.parse_iterations(logref)[-3:], flags)


@pytest.mark.gpu
def test_gpu_two_vector_device_memory(tmp_path):
    """The 2-vector solver holds r, d, the reduction accumulator and the per-step sums only."""
    from chfem_b200 import _native
    from tests.test_gpu_parity import host_arrays
    spec = fixture()["cases"]["pore16"]["spec"]
    nf, raw = make_case(tmp_path, "pore16", spec)
    a = host_arrays(nf, raw)
    lib = _native.cudapcg()
    lib.cudapcgB200DeviceBytes.restype = ctypes.c_ulonglong
    sizes = {}
    for solver in (1, 5):
        _native.setup_cudapcg_model(lib, a)
        assert lib.cudapcgSetSolver(solver)
        assert lib.cudapcgAllocateArrays()
        sizes[solver] = lib.cudapcgB200DeviceBytes()
        lib.cudapcgEnd()
    maps = 4 * a["N"] + 4 * (a["nV"] + a["nB"]) + a["nB"]
    assert sizes[5] == maps + 16 * a["ndof"]  # the accumulators come with the first solve
    assert sizes[1] > maps + 7 * 8 * a["ndof"]


@pytest.mark.gpu
def test_gpu_compute_property_minres2():
    from chfem_b200 import compute_property
    from chfem_b200.synthetic import pore_grf
    img = pore_grf((14, 16, 12), corr=2.0, porosity=0.5, seed=3)
    K1 = compute_property("permeability", img, solver="minres", solver_tolerance=1e-9)
    K2 = compute_property("permeability", img, solver="minres2", solver_tolerance=1e-9)
    K3 = compute_property("permeability", img, solver="cg2", solver_tolerance=1e-9)
    assert H.rel_to_max(K2, K1) < 1e-6 and H.rel_to_max(K3, K1) < 1e-6
    with pytest.raises(ValueError, match="Two-vectors"):
        compute_property("conductivity", img, {0: 1.0, 255: 2.0}, solver="cg2")
