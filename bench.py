#!/usr/bin/env python
"""bench.py -- time-to-tolerance of chfem_b200 on one B200 (or N, one process per GPU).

Workload (default): linear elasticity, 128^3 uint8 image, two phases from a periodic Gaussian
random field (correlation length 6 voxels, seed 2000) thresholded to 40 % phase 1;
E/nu = 1.0/0.30 and 10.0/0.20; six load cases -> 6x6 stiffness; Jacobi PCG to the relative
residual sqrt(r'M^-1 r / r0'M^-1 r0) <= 1e-6; mixed precision (FP32 fields and operator,
FP64 reductions, residual replacement every 50 iterations).  6 291 456 DOF.  Synthetic data
(no datasets offline).

A step is one homogenization of the workload (all load cases solved to tolerance).
  value     device time of a step with the model resident in HBM (CUDA events around each
            solve inside the library; RHS uploads excluded), max over ranks;
  e2e       the same through the public API (compute_property's native entry chfemB200Run):
            host image in, tensor out -- maps, uploads, solves, downloads, tensor updates.
Per-GPU work is fixed as N grows (each rank solves its own sample, seed 2000 + rank): weak.

--impl reference runs the reference's own CUDA build (oracle/_ref/chfem_exec_ref, compiled
from its sources for sm_100a, stock FP64 path) on the same workload on this GPU.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "elastic128_grf_mixed": dict(analysis=1, shape=(128, 128, 128), gen="grf", corr=6.0, fraction=0.40, seed=2000,
                                 props={0: (1.0, 0.30), 255: (10.0, 0.20)}, tol=1e-6, maxit=20000, precision="mixed"),
    "elastic128_grf_fp64": dict(analysis=1, shape=(128, 128, 128), gen="grf", corr=6.0, fraction=0.40, seed=2000,
                                props={0: (1.0, 0.30), 255: (10.0, 0.20)}, tol=1e-6, maxit=20000, precision="fp64"),
    "elastic256_grf_mixed_block": dict(analysis=1, shape=(256, 256, 256), gen="grf", corr=6.0, fraction=0.40, seed=5000,
                                       props={0: (1.0, 0.30), 255: (10.0, 0.20)}, tol=1e-6, maxit=20000,
                                       precision="mixed", multirhs=True),
    "elastic256_grf_mixed_block_learned": dict(analysis=1, shape=(256, 256, 256), gen="grf", corr=6.0, fraction=0.40,
                                               seed=5000, props={0: (1.0, 0.30), 255: (10.0, 0.20)}, tol=1e-6,
                                               maxit=20000, precision="mixed", multirhs=True, learned=True),
    "elastic128_grf_mixed_block_learned": dict(analysis=1, shape=(128, 128, 128), gen="grf", corr=6.0, fraction=0.40,
                                               seed=2000, props={0: (1.0, 0.30), 255: (10.0, 0.20)}, tol=1e-6,
                                               maxit=20000, precision="mixed", multirhs=True, learned=True),
    "thermal64_spheres_fp64": dict(analysis=0, shape=(64, 64, 64), gen="spheres", vf=0.30, seed=1000,
                                   props={0: 1.0, 255: 10.0}, tol=1e-6, maxit=20000, precision="fp64"),
    "elastic128_grf_mixed_block": dict(analysis=1, shape=(128, 128, 128), gen="grf", corr=6.0, fraction=0.40, seed=2000,
                                       props={0: (1.0, 0.30), 255: (10.0, 0.20)}, tol=1e-6, maxit=20000,
                                       precision="mixed", multirhs=True),
    # the thermal operator above L2 (256^3: 16.8 M nodes, 570 MB per FP64 operator pass);
    # overlapping balls (non-overlapping placement jams below 0.30 at this size)
    "thermal256_spheres_fp64": dict(analysis=0, shape=(256, 256, 256), gen="spheres", vf=0.30, seed=1100, overlap=True,
                                    props={0: 1.0, 255: 10.0}, tol=1e-6, maxit=20000, precision="fp64"),
    "thermal256_spheres_mixed": dict(analysis=0, shape=(256, 256, 256), gen="spheres", vf=0.30, seed=1100, overlap=True,
                                     props={0: 1.0, 255: 10.0}, tol=1e-6, maxit=20000, precision="mixed"),
    "thermal64_spheres_fp64_block": dict(analysis=0, shape=(64, 64, 64), gen="spheres", vf=0.30, seed=1000,
                                         props={0: 1.0, 255: 10.0}, tol=1e-6, maxit=20000, precision="fp64",
                                         multirhs=True),
    # Stokes solves run in FP64 in every precision mode (the (P)MINRES recurrence nears breakdown
    # on the indefinite system, where FP32 rounding stalls it)
    "stokes128_grf_fp64": dict(analysis=2, shape=(128, 128, 128), gen="pore", corr=8.0, porosity=0.35, seed=3000,
                               props=None, tol=1e-6, maxit=100000, precision="fp64", solver=1),
    "stokes128_grf_fp64_block": dict(analysis=2, shape=(128, 128, 128), gen="pore", corr=8.0, porosity=0.35, seed=3000,
                                     props=None, tol=1e-6, maxit=100000, precision="fp64", solver=1, multirhs=True),
    # 512 independent sphere-inclusion images, edge uniform in {32, 48, 64, 96}, volume fraction
    # U[0.1, 0.5] (overlapping balls of radius 4-8), k1/k0 log-uniform in [2, 100], 3 load cases
    # each, all solved in one device-resident batch
    "thermal_batch512_mixed": dict(analysis=0, batch=512, edges=(32, 48, 64, 96), seed=4000, tol=1e-6, maxit=10000,
                                   precision="mixed"),
    "thermal_batch512_fp64": dict(analysis=0, batch=512, edges=(32, 48, 64, 96), seed=4000, tol=1e-6, maxit=10000,
                                  precision="fp64"),
}
DEFAULT = "elastic128_grf_mixed_block_learned"


def make_image(w, rank):
    from chfem_b200 import synthetic
    seed = w["seed"] + rank
    if w["gen"] == "grf":
        return synthetic.grf(w["shape"], corr=w["corr"], fraction=w["fraction"], seed=seed)
    if w["gen"] == "spheres":
        return synthetic.spheres(w["shape"], vf=w["vf"], seed=seed, overlap=w.get("overlap", False))
    return synthetic.pore_grf(w["shape"], corr=w["corr"], porosity=w["porosity"], seed=seed)


def write_case(wd, w, img, tol=None, maxit=None):
    from chfem_b200.io import export_for_chfem
    prefix = os.path.join(wd, "case")
    export_for_chfem(prefix + ".raw", img, w["analysis"], mat_props=w["props"], voxel_size=1.0,
                     solver_type=w.get("solver", 0), solver_tolerance=tol or w["tol"],
                     solver_maxiter=maxit or w["maxit"])
    return prefix + ".nf", prefix + ".raw"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9 or (vis.isdigit() and f[0] != vis):
                    continue
                sm.append(float(f[1]))
                smax = float(f[2])
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except Exception:
            pass
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------
class Resident:
    """The workload's model resident on the GPU through the cudapcg C ABI; one step solves
    every load case (RHS assembled once on the host, uploaded per case)."""

    def __init__(self, nf, raw, w):
        from chfem_b200 import _native
        from chfem_b200._native import setup_cudapcg_model as setup_model
        self.h = _native.chfem()
        self.c = _native.cudapcg()
        self.h.chfemB200SetQuiet(1)
        assert self.h.hmgInit(nf.encode(), raw.encode(), None, None), self.h.chfemB200LastError()
        info = (ctypes.c_uint * 9)()
        self.h.chfemB200ModelInfo(info)
        self.info = list(info)
        self.ndof = info[4]
        self.N = info[3]
        self.analysis = info[8]
        ncases = 6 if self.analysis == 1 else 3
        self.rhs = []
        for d in range(ncases):
            r = np.zeros(self.ndof)
            self.h.chfemB200AssembleRHS(d, r.ctypes.data_as(ctypes.c_void_p))
            self.rhs.append(r)

        def arr(wh, t):
            n = self.h.chfemB200ModelArraySize(wh)
            x = np.zeros(n // np.dtype(t).itemsize, dtype=t)
            if n:
                self.h.chfemB200CopyModelArray(wh, x.ctypes.data_as(ctypes.c_void_p), n)
            return x
        a = dict(nx=info[0], ny=info[1], nz=info[2], N=info[3], ndof=info[4], nV=info[5], nB=info[6],
                 nkeys=info[7] if info[8] != 2 else 1, analysis=info[8], keys=arr(0, np.uint16),
                 dof_of_node=arr(1, np.uint32), node_of_dof=arr(2, np.uint32), border=arr(3, np.uint8),
                 lcl=arr(4, np.float64))
        self.CB = arr(7, np.float64)
        self.lcl_size = int(a["lcl"].size)
        self.nmat = int(a["nkeys"])
        self.dims = (info[0], info[1], info[2])
        setup_model(self.c, a)
        self.c.cudapcgSetSolver(w.get("solver", 0))
        self.c.cudapcgSetPreconditioner(1)
        self.c.cudapcgSetNumTol(ctypes.c_double(w["tol"]))
        self.c.cudapcgSetMaxIterations(w["maxit"])
        self.set_precision(w["precision"])
        self.x = np.zeros(self.ndof)

    def set_precision(self, p):
        self.c.cudapcgB200SetPrecision(1 if p == "mixed" else 0)
        assert self.c.cudapcgAllocateArrays()

    def step(self, multirhs=False):
        from chfem_b200._native import CudapcgStats
        if multirhs:  # every load case in one block solve
            nr = len(self.rhs)
            if not hasattr(self, "xs"):
                self.xs = [np.zeros(self.ndof) for _ in range(nr)]
            P = ctypes.c_void_p * nr
            prhs = P(*[r.ctypes.data for r in self.rhs])
            px = P(*[x.ctypes.data for x in self.xs])
            its = (ctypes.c_uint * nr)()
            res = (ctypes.c_double * nr)()
            self.c.cudapcgB200SolveBlock(nr, prhs, None, 0, px, its, res)
            err = self.c.cudapcgB200LastError()
            assert not err, err
            st = CudapcgStats()
            self.c.cudapcgB200GetStats(ctypes.byref(st))
            return st.solve_seconds + st.setup_seconds, list(its), st.kernel_launches
        dev, its, launches = 0.0, [], 0
        for r in self.rhs:
            self.c.cudapcgSetRHS(r.ctypes.data_as(ctypes.c_void_p))
            self.c.cudapcgSolve(self.x.ctypes.data_as(ctypes.c_void_p))
            st = CudapcgStats()
            self.c.cudapcgB200GetStats(ctypes.byref(st))
            dev += st.solve_seconds + st.setup_seconds
            its.append(st.iterations)
            launches += st.kernel_launches
        return dev, its, launches

    def step_learned(self, img, props):
        """All six load cases from the trained network's guesses: device time of the network
        (CUDA events on its stream) plus the block solve (cudapcgB200SolveLoadCases, device x0)."""
        import torch
        from chfem_b200 import learned
        from chfem_b200._native import CudapcgStats
        net = learned.default_net()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        xs = learned.device_guesses(net, img, props)
        e1.record()
        torch.cuda.synchronize()
        t_net = e0.elapsed_time(e1) * 1e-3
        P = ctypes.c_void_p * 6
        axis = (ctypes.c_int * 6)(*learned.CASE_AXIS)
        comp = (ctypes.c_int * 6)(*learned.CASE_COMP)
        jump = (ctypes.c_double * 6)(*[float(self.dims[a]) for a in learned.CASE_AXIS])
        vol = np.zeros(36)
        its = (ctypes.c_uint * 6)()
        res = (ctypes.c_double * 6)()
        self.c.cudapcgB200SolveLoadCases(6, axis, comp, jump, self.CB.ctypes.data_as(ctypes.c_void_p), 6,
                                         P(*[x.data_ptr() for x in xs]), 2, vol.ctypes.data_as(ctypes.c_void_p), None, its, res)
        err = self.c.cudapcgB200LastError()
        assert not err, err
        st = CudapcgStats()
        self.c.cudapcgB200GetStats(ctypes.byref(st))
        return t_net + st.solve_seconds + st.setup_seconds, list(its), st.kernel_launches + 40, t_net

    def kernel_time(self, which, reps=20):
        self.c.cudapcgB200TimeKernel.restype = ctypes.c_double
        return self.c.cudapcgB200TimeKernel(which, reps)

    def close(self):
        self.c.cudapcgEnd()
        self.h.hmgEnd()


def kernel_only(w, workload, which):
    """One kernel of the workload's model launched 10 times after warm-up, its mean CUDA-event time
    printed: the command the ncu captures under profiles/ run."""
    img = make_image(w, 0)
    wd = tempfile.mkdtemp()
    nf, raw = write_case(wd, w, img)
    m = Resident(nf, raw, w)
    t = m.kernel_time(which, reps=10)
    print(json.dumps({"workload": workload, "kernel": which, "ms": t * 1e3, "nodes": m.N, "ndof": m.ndof}))
    m.close()


def e2e_step(img, nf, w):
    """One homogenization through the public API's native entry (compute_property's path)."""
    from chfem_b200 import _native
    if w.get("learned"):
        from chfem_b200 import compute_property
        t0 = time.perf_counter()
        C = np.array(compute_property("elasticity", img, mat_props=w["props"], voxel_size=1.0, solver_tolerance=w["tol"],
                                      solver_maxiter=w["maxit"], precision=w["precision"], multirhs=True,
                                      initial_guess="learned"))
        return time.perf_counter() - t0, C, _native.solve_stats()
    lib = _native.chfem()
    lib.chfemB200SetQuiet(1)
    flat = np.ascontiguousarray(img.reshape(-1))
    C = np.zeros(36)
    t0 = time.perf_counter()
    n = lib.chfemB200Run(flat.ctypes.data_as(ctypes.c_void_p), nf.encode(), 6, w.get("solver", 0), 1,
                         1 if w["precision"] == "mixed" else 0, int(w.get("multirhs", False)),
                         C.ctypes.data_as(ctypes.c_void_p))
    t = time.perf_counter() - t0
    assert n, lib.chfemB200LastError()
    st = _native.solve_stats()
    return t, C[: n * n].reshape(n, n), st


def cpu_baseline(nf_dir, w, img, total_iters):
    """The oracle (reference host code + CPU restatement of its solver) on the host cores: a
    bounded sample of the workload (one load case, a fixed number of iterations), scaled to
    the full job by the iteration count of the FP64 solve."""
    exe = os.path.join(ROOT, "oracle", "_ref", "chfem_oracle_exec")
    if not os.path.exists(exe):
        return None
    sample_its = 30 if w["analysis"] == 1 else 200
    nf, raw = write_case(nf_dir, w, img, tol=1e-30, maxit=sample_its)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    p = subprocess.run([exe, nf, raw, "-d", "0"], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, OMP_NUM_THREADS=str(cores)))
    wall = time.perf_counter() - t0
    per_it = None
    for line in p.stdout.splitlines():
        if "Mean time per iteration" in line:
            per_it = float(line.split(":")[1].split()[0])
    if per_it is None:
        return None
    return {"value": per_it * total_iters, "unit": "s", "cores": cores, "kind": "port",
            "sample": f"oracle CPU FP64 PCG, load case X, {sample_its} iterations ({wall:.1f} s wall), "
                      f"{per_it:.3e} s/iteration x {total_iters} iterations of the full FP64 job"}


# ---------------------------------------------------------------------------------------
# Batched thermal workload (independent samples, one batch solve per step)
def make_batch(w, rank):
    from chfem_b200 import synthetic
    rng = np.random.default_rng(w["seed"] + 7919 * rank)
    imgs, props = [], []
    for i in range(w["batch"]):
        e = int(rng.choice(w["edges"]))
        vf = float(rng.uniform(0.1, 0.5))
        ratio = float(np.exp(rng.uniform(np.log(2.0), np.log(100.0))))
        imgs.append(synthetic.spheres((e, e, e), vf=vf, seed=w["seed"] + i + 100000 * rank, overlap=True))
        props.append({0: 1.0, 255: ratio})
    return imgs, props


def batch_cpu_rate(imgs, props, w, exe, budget_s=20.0):
    """Seconds per node-iteration of a solver CLI (oracle or reference build) on the smallest
    samples of the batch, each homogenized in full (3 load cases), until budget_s is spent."""
    from chfem_b200.io import export_for_chfem
    order = sorted(range(len(imgs)), key=lambda i: imgs[i].size)
    t_sum, ni_sum, done, walls = 0.0, 0, 0, 0.0
    with tempfile.TemporaryDirectory() as d:
        for i in order[:8]:
            nf = os.path.join(d, f"s{i}.nf")
            export_for_chfem(os.path.join(d, f"s{i}.raw"), imgs[i], 0, mat_props=props[i], voxel_size=1.0,
                             solver_tolerance=w["tol"], solver_maxiter=w["maxit"])
            t0 = time.perf_counter()
            p = subprocess.run([exe, nf, os.path.join(d, f"s{i}.raw")], capture_output=True, text=True, timeout=600, cwd=d)
            wall = time.perf_counter() - t0
            if p.returncode != 0:
                return None
            its = [int(l.split("iteration:")[1].split(",")[0]) for l in p.stdout.splitlines() if "iteration:" in l and "residual" in l]
            solve = sum(float(l.split(":")[1].split()[0]) for l in p.stdout.splitlines() if "| Elapsed time:" in l)
            t_sum += solve if solve > 0 else wall
            walls += wall
            ni_sum += imgs[i].size * sum(its)
            done += 1
            if walls > budget_s:
                break
    if not ni_sum:
        return None
    return t_sum / ni_sum, walls / ni_sum, done


def batch_main(args, w, world, rank, dist, allmax, barrier):
    from chfem_b200 import compute_conductivity_batch, _native
    imgs, props = make_batch(w, rank)
    nodes = int(sum(a.size for a in imgs))

    def step():
        t0 = time.perf_counter()
        C, its = compute_conductivity_batch(imgs, props, solver_tolerance=w["tol"], solver_maxiter=w["maxit"],
                                            precision=w["precision"], return_iterations=True)
        wall = time.perf_counter() - t0
        st = _native.batch_stats()
        return C, its, st, wall

    first = None
    for k in range(args.warmup):
        r = step()
        first = first or r
    clocks = Clocks()
    barrier()
    clocks.start()
    dev, walls, launches = [], [], 0
    for _ in range(args.steps):
        C, its, st, wall = step()
        dev.append(st.setup_seconds + st.solve_seconds)
        walls.append(wall)
        launches += st.kernel_launches
    barrier()
    clk = clocks.stop()
    step_s = allmax(float(np.mean(dev)))
    e2e = allmax(float(np.mean(walls)))
    st0 = first[2] if first else st
    es = 4 if w["precision"] == "mixed" else 8
    per_unit = 12 * es + 2
    peak, peak_kind = load_peaks()
    tile = {4: 0, 8: 1, 16: 2}.get(st0.tile_cols, 1)
    kt = st0.tile_ms[tile] * 1e-3 if st0.tile_ms[tile] > 0 else None
    achieved = per_unit * nodes / kt / 1e9 if kt else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "traffic": profiled_traffic(args.workload),
                "kernel": f"k_bt_apply<{st0.tile_cols},{'float' if es == 4 else 'double'},false> (batch operator + directions + dots, "
                          f"{w['batch']} samples x 3 load cases; tile 32x{st0.tile_cols} chosen by the autotuner)",
                "kernel_ms": kt * 1e3 if kt else None, "bytes_per_unit": per_unit, "units_per_launch": nodes,
                "tile_ms_4_8_16": list(st0.tile_ms), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}
    node_its = float(sum(imgs[i].size * int(its[i].sum()) for i in range(len(imgs))))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        exe = os.path.join(ROOT, "oracle", "_ref", "chfem_oracle_exec")
        if os.path.exists(exe):
            r = batch_cpu_rate(imgs, props, w, exe)
            if r:
                cpu = {"value": r[0] * node_its, "unit": "s", "cores": os.cpu_count() or 1, "kind": "port",
                       "sample": f"oracle CPU FP64 PCG on the {r[2]} smallest samples, all load cases: "
                                 f"{r[0]:.3e} s per node-iteration x {node_its:.3e} node-iterations of the batch"}
    if rank == 0:
        line = {"metric": metric_name(w), "value": step_s, "unit": "s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64" if es == 4 else "f64", "data": "synthetic",
                "config": config_dict(args, w, world) | {"samples": w["batch"], "nodes": nodes},
                "iterations_max": int(its.max()), "iterations_mean": float(its.mean()),
                "dof_iterations_per_s": node_its / step_s, "samples_per_s": world * w["batch"] / step_s,
                "roofline": roofline, "clocks": clk, "gpu_launches": int(launches),
                "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": int(3 * nodes),
                        "d2h_bytes_per_step": int(w["batch"] * 9 * 8 + w["batch"] * 3 * 4),
                        "path": "compute_conductivity_batch (images in host memory -> tensors)"},
                "cpu_baseline": cpu}
        print(json.dumps(line))


def reference_batch(args, w):
    """Reference arm of a batch workload: the reference's CUDA build run image by image (its only
    way) on the smallest samples for a bounded time, scaled by node-iterations to the batch."""
    exe = os.path.join(ROOT, "oracle", "_ref", "chfem_exec_ref")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "reference CUDA build oracle/_ref/chfem_exec_ref not built"}))
        return
    imgs, props = make_batch(w, 0)
    from chfem_b200 import compute_conductivity_batch
    C, its = compute_conductivity_batch(imgs, props, solver_tolerance=w["tol"], solver_maxiter=w["maxit"], precision="fp64",
                                        return_iterations=True)
    node_its = float(sum(imgs[i].size * int(its[i].sum()) for i in range(len(imgs))))
    vals, walls = [], []
    for _ in range(max(1, args.steps)):
        r = batch_cpu_rate(imgs, props, w, exe, budget_s=30.0)
        if not r:
            print(json.dumps({"impl": "reference", "unavailable": "reference run failed"}))
            return
        vals.append(r[0] * node_its)
        walls.append(r[1] * node_its)
    v = float(np.mean(vals))
    line = {"metric": metric_name(w), "value": v, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference", "config": config_dict(args, w, 1) | {"samples": w["batch"]},
            "cpu_baseline": {"value": v, "unit": "s", "cores": 0, "kind": "reference",
                             "sample": f"reference CUDA build, one process per image, on the {r[2]} smallest samples, "
                                       "its solver time per node-iteration scaled to the batch's node-iterations"},
            "e2e": {"value": float(np.mean(walls)), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def reference_arm(args, w):
    exe = os.path.join(ROOT, "oracle", "_ref", "chfem_exec_ref")
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "reference CUDA build oracle/_ref/chfem_exec_ref not built"}))
        return
    img = make_image(w, 0)
    ncase = 6 if w["analysis"] == 1 else 3
    ndof = img.size * (3 if w["analysis"] == 1 else 1) if w["analysis"] != 2 else None
    if ndof:  # stock FP64 path: 2-byte keys, element matrices; per load case RHS up and x down
        h2d = int(2 * img.size + 8 * 2 * 576 + ncase * 8 * ndof)
        d2h = int(ncase * 8 * ndof)
    else:
        h2d, d2h = None, None
    with tempfile.TemporaryDirectory() as wd:
        nf, raw = write_case(wd, w, img)
        times, walls, its = [], [], []
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            p = subprocess.run([exe, nf, raw, "-d", "6"], capture_output=True, text=True, timeout=3000, cwd=wd)
            wall = time.perf_counter() - t0
            if p.returncode != 0:
                print(json.dumps({"impl": "reference", "unavailable": "reference run failed: " + p.stdout[-200:].replace("\n", " ")}))
                return
            solve = sum(float(l.split(":")[1].split()[0]) for l in p.stdout.splitlines() if "| Elapsed time:" in l)
            it = [int(l.split("iteration:")[1].split(",")[0]) for l in p.stdout.splitlines()
                  if "iteration:" in l and "residual" in l]
            if k >= args.warmup:
                times.append(solve)
                walls.append(wall)
                its = it
        v = float(np.mean(times))
        line = {"metric": metric_name(w), "value": v, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": config_dict(args, w, 1) | {"precision": "fp64", "multirhs": False, "initial_guess": "zero",
                                                     "reference_build": "stock FP64, 16-bit keys, 128 threads/block, sm_100a"},
                "iterations": its,
                "cpu_baseline": {"value": v, "unit": "s", "cores": os.cpu_count() or 1, "kind": "reference",
                                 "sample": "the reference's CUDA build on the same B200 (its only solver path: it has no CPU "
                                           "solver), full workload; host threads = its OpenMP host code"},
                "e2e": {"value": float(np.mean(walls)), "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "path": "chfem_exec process wall time (files in, tensor out); copies: node keys, element matrices, "
                                "and per load case its right-hand side up and its solution down"}}
        print(json.dumps(line))


def profiled_traffic(workload):
    """DRAM bytes (read + write) per launch of the dominant kernel, from the ncu summaries in
    profiles/ (lines "dram_bytes_per_launch: <workload> <bytes>"); None when not captured."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith(".md"):
            continue
        with open(os.path.join(pdir, fn)) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 3 and parts[0] == "dram_bytes_per_launch:" and parts[1] == workload:
                    return int(parts[2])
    return None


def metric_name(w):
    if "batch" in w:
        return "time-to-tol 1e-6 (s): all samples x 3 load cases of the batch, device time"
    return "time-to-tol 1e-6 (s): all load cases of the workload, device time, model resident"


def config_dict(args, w, n):
    if "batch" in w:
        return {"workload": args.workload, "samples": w["batch"], "edges": list(w["edges"]), "analysis": "thermal",
                "load_cases": 3, "tol": w["tol"], "precision": w["precision"], "solver": "PCG", "preconditioner": "Jacobi",
                "images": "overlapping balls r 4-8, vf U[0.1,0.5], k1/k0 log-U[2,100]",
                "l2": "working set > L2 (the batch's vectors total GBs)", "parallelism": f"samples x{n}"}
    return {"workload": args.workload, "shape_zyx": list(w["shape"]), "analysis": ["thermal", "elastic", "stokes"][w["analysis"]],
            "load_cases": 6 if w["analysis"] == 1 else 3, "tol": w["tol"], "precision": w["precision"],
            "solver": "PMINRES" if w.get("solver", 0) == 1 else "PCG", "preconditioner": "Jacobi",
            "multirhs": bool(w.get("multirhs", False)), "initial_guess": "learned" if w.get("learned") else "zero",
            "l2": "working set > L2 (vectors of the elastic 128^3 case ~25-50 MB each)", "parallelism": f"samples x{n}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-check", action="store_true", help="skip the untimed reference run (tensor error, same-precision ratio)")
    ap.add_argument("--no-elastic256", action="store_true", help="skip the 256^3 elastic sub-record of the default workload")
    ap.add_argument("--kernel", type=int, default=None,
                    help="only time one kernel of the workload's resident model, 10 launches (for ncu captures): "
                         "0 plain operator pass, 1 operator pass (PCG), 2 pointwise pass (PCG), 3 operator pass "
                         "((P)MINRES), 5 block operator pass, 6 block pointwise pass")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.kernel is not None:
        kernel_only(w, args.workload, args.kernel)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:  # one GPU per process: pin before any CUDA context exists
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = vis.split(",") if vis else [str(i) for i in range(64)]
        os.environ["CUDA_VISIBLE_DEVICES"] = devs[local]
    if args.impl == "reference":
        if "batch" in w:
            if rank == 0:
                reference_batch(args, w)
            return
        reference_arm(args, w)
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(0)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist

    def barrier():
        if dist:
            dist.barrier()

    def allmax(v):
        if not dist:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if "batch" in w:
        batch_main(args, w, world, rank, dist, allmax, barrier)
        if dist:
            dist.destroy_process_group()
        return
    img = make_image(w, rank)
    wd = tempfile.mkdtemp()
    nf, raw = write_case(wd, w, img)
    model = Resident(nf, raw, w)
    # plain FP64 PCG time-to-tol for comparison (once, outside the timed region)
    fp64 = None
    block = bool(w.get("multirhs", False))
    if w["precision"] == "mixed" or block:
        model.set_precision("fp64")
        t64, its64, _ = model.step()
        fp64 = {"time_s": t64, "iterations": its64}
        model.set_precision(w["precision"])
    learned_run = bool(w.get("learned"))
    net_times = []

    def run_step():
        if learned_run:
            d, its_, l_, tn = model.step_learned(img, w["props"])
            net_times.append(tn)
            return d, its_, l_
        return model.step(block)
    zero_guess = None
    if learned_run:  # the same block solve from the zero guess, for the iteration comparison
        zero_guess = {"time_s": model.step(block)[0], "iterations": model.step(block)[1]}
    for _ in range(args.warmup):
        run_step()
    clocks = Clocks()
    barrier()
    clocks.start()
    t0 = time.perf_counter()
    dev_total, its, launches = 0.0, None, 0
    for _ in range(args.steps):
        d, its, l = run_step()
        dev_total += d
        launches += l
    wall = time.perf_counter() - t0
    barrier()
    clk = clocks.stop()
    step_s = allmax(dev_total / args.steps)
    wall_step = allmax(wall / args.steps)
    dev_bytes = int(model.c.cudapcgB200DeviceBytes())
    roofline = dominant_kernel_roofline(model, w, block, args.workload)
    total_its = sum(its)
    dof_its = model.ndof * total_its / (dev_total / args.steps)
    # e2e through the public API (host image in, tensor out): one untimed call, then the mean of
    # as many calls as timed steps, like the device-time value
    e2e_step(img, nf, w)
    e2e_times, breakdowns = [], []
    C = None
    for k in range(args.steps):
        t, C, st = e2e_step(img, nf, w)
        ncs = max(1, st.n_cases)
        breakdowns.append([t - st.total_seconds, st.rhs_seconds, float(sum(st.solve_seconds[i] for i in range(ncs))),
                           st.update_seconds, st.setup_seconds, st.total_seconds, st.solve_call_seconds, st.teardown_seconds])
        e2e_times.append(t)
    bm = np.mean(np.array(breakdowns), axis=0)
    breakdown = {"model_build_and_upload_s": bm[0], "rhs_assembly_s": bm[1], "solve_device_s": bm[2],
                 "tensor_update_s": bm[3], "solver_setup_s": bm[4], "solver_call_total_s": bm[5],
                 "solve_calls_wall_s": bm[6], "teardown_s": bm[7]}
    e2e = allmax(float(np.mean(e2e_times)))
    # the plain method end to end (FP64, one load case at a time, zero guess): its tensor is the
    # FP64 reference of the mixed / block / learned one
    plain_e2e, Cp = None, None
    if w["precision"] == "mixed" or block or learned_run:
        from chfem_b200 import _native as _nat
        lib = _nat.chfem()
        lib.chfemB200SetQuiet(1)
        flat = np.ascontiguousarray(img.reshape(-1))
        Cp = np.zeros(36)
        t0 = time.perf_counter()
        n = lib.chfemB200Run(flat.ctypes.data_as(ctypes.c_void_p), nf.encode(), 6, w.get("solver", 0), 1, 0, 0,
                             Cp.ctypes.data_as(ctypes.c_void_p))
        plain_e2e = allmax(time.perf_counter() - t0)
        Cp = Cp[: n * n].reshape(n, n)
    ncase = 6 if w["analysis"] == 1 else 3
    ns = 6 if w["analysis"] == 1 else 3
    # copies of one call: the 1-byte image (node keys are built on the device from it; Stokes
    # pore maps on the host), the element matrices and tensor matrices, and out the volume-term
    # moments of every load case
    maps = 9 * model.N if w["analysis"] == 2 else 0
    h2d = int(img.size + maps + 8 * (model.lcl_size + model.CB.size))
    d2h = int(ncase * ns * 8)
    model.close()
    cpu, ref = None, None
    if rank == 0 and world == 1:
        if not args.no_cpu_baseline:
            its64 = sum(fp64["iterations"]) if fp64 else total_its
            cpu = cpu_baseline(wd, w, img, its64)
        if not args.no_reference_check:
            ref = reference_once(wd, w, img)
    if rank == 0:
        line = {"metric": metric_name(w), "value": step_s, "unit": "s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64" if w["precision"] == "mixed" else "f64", "data": "synthetic",
                "config": config_dict(args, w, world),
                "iterations": its, "dof_iterations_per_s": dof_its, "wall_s_per_step": wall_step,
                "plain_fp64_pcg": fp64, "speedup_vs_plain_fp64": (fp64["time_s"] / step_s) if fp64 else None,
                "tensor_diag": [float(C[i, i]) for i in range(C.shape[0])] if C is not None else None,
                "roofline": roofline, "clocks": clk, "gpu_launches": int(launches),
                "device_bytes_per_dof": dev_bytes / model.ndof,
                "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "path": ("compute_property(..., initial_guess='learned')" if learned_run else
                                 "chfemB200Run (compute_property's native entry)") + ": image in host memory -> tensor; "
                                f"mean of {args.steps} calls after one untimed call",
                        "breakdown": breakdown},
                "cpu_baseline": cpu, "samples_per_s": world / step_s}
        if Cp is not None and C is not None:
            line["tensor_rel_err_vs_plain_fp64"] = rel_to_max(C, Cp)
        if plain_e2e is not None:
            line["plain_fp64_e2e_s"] = plain_e2e
            line["e2e_speedup_vs_plain_fp64"] = plain_e2e / e2e
        if ref is not None:
            line["reference_check"] = ref
            if C is not None and ref.get("C") is not None:
                line["tensor_rel_err_vs_reference"] = rel_to_max(C, np.array(ref["C"]))
            if fp64 and ref.get("solve_s"):
                line["same_precision_ratio"] = ref["solve_s"] / fp64["time_s"]
        if learned_run:
            line["learned_guess"] = {"network_s": float(np.mean(net_times[-args.steps:])), "zero_guess_block": zero_guess,
                                     "weights": "chfem_b200/weights/elastic_unet.bin"}
        if rank == 0 and world == 1 and not args.no_elastic256 and args.workload == DEFAULT:
            line["elastic256"] = elastic256_record()
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def rel_to_max(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def dominant_kernel_roofline(model, w, block, workload):
    """The dominant kernel timed live on the library's stream (CUDA events around each launch),
    its algorithmic bytes per node against the measured HBM peak."""
    peak, peak_kind = load_peaks()
    es = 4 if w["precision"] == "mixed" else 8
    if w["analysis"] == 2:
        kern_which, kname = 3, "k_fl_apply<MR> (Stokes operator + PMINRES step, one right-hand side)"
        # per DOF: r, q, d in, q', r' out (5 es) and the FP64 x read and written (16 B); per row
        # set (pore node: 4 DOFs, interface node: 1) its DOF->node and node->DOF entries (8 B) and
        # an interface node's fluid key (1 B); units = row sets, bytes_per_unit their mean
        nV, nB = model.info[5], model.info[6]
        units = nV + nB
        per_unit = (nV * (4 * (5 * es + 16) + 8) + nB * ((5 * es + 16) + 9)) / max(1, units)
    else:
        nd = 3 if w["analysis"] == 1 else 1
        tn = 'float' if es == 4 else 'double'
        if block:
            nr = 6 if nd == 3 else 3
            asm = model.nmat <= 2 and os.environ.get("CHFEM_B200_BLOCK_OP") != "element"
            kern_which = 5
            kname = (f"k_asm_apply<{nd},{tn},{nr}> (block operator, stencil assembled per material configuration, "
                     f"+ directions + dots, {nr} load cases)" if asm else
                     f"k_blk_apply<{nd},{tn},{nr}> (block operator + directions + dots, {nr} load cases)")
            per_unit = nr * 4 * nd * es + 2  # per load case s, d_old in; d_new, q out; one 16-bit key
        elif nd == 1 and model.nmat <= 4 and os.environ.get("CHFEM_B200_THERMAL_OP") != "generic":
            kern_which = 1
            kname = f"k_th_apply<{tn},TE_PCG> (thermal operator for cubic-symmetric conduction matrices + direction + dot)"
            per_unit = 4 * es + 2
        else:
            kern_which, kname = 1, f"k_te_apply<{nd},{tn},TE_PCG> (operator + direction + dot)"
            per_unit = 4 * nd * es + 2  # s, d_old in; d_new, q out (nd comps); 16-bit key
        units = model.N
    kt = model.kernel_time(kern_which, reps=30)
    achieved = per_unit * units / kt / 1e9 if kt > 0 else None
    # FP work of the operator as the reference formulates it (64 element blocks per node)
    fl_unit = (1152 if w["analysis"] == 1 else 80) * ((6 if w["analysis"] == 1 else 3) if block else 1)
    flops = fl_unit * units / kt / 1e12 if (kt > 0 and w["analysis"] != 2) else None
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "traffic": profiled_traffic(workload),
            "kernel": kname, "kernel_ms": kt * 1e3, "bytes_per_unit": per_unit, "units_per_launch": units,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
            "fp_tflops_reference_formulation": flops}


def reference_once(wd, w, img):
    """One run of the reference's CUDA build (stock FP64, one load case at a time) on the same
    workload, outside the timed region: its tensor (for the tensor error of this line) and its
    summed solver times (for the same-precision ratio against this library's plain FP64 PCG)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "chfem_exec_ref")
    if not os.path.exists(exe):
        return None
    nf, raw = write_case(wd, w, img)
    out = os.path.join(wd, "ref_C.bin")
    p = subprocess.run([exe, nf, raw, "-d", "6", "-b", out], capture_output=True, text=True, timeout=3000, cwd=wd)
    if p.returncode != 0 or not os.path.exists(out):
        return {"error": p.stdout[-200:]}
    C = np.fromfile(out)
    k = int(round(np.sqrt(C.size)))
    solve = sum(float(l.split(":")[1].split()[0]) for l in p.stdout.splitlines() if "| Elapsed time:" in l)
    its = [int(l.split("iteration:")[1].split(",")[0]) for l in p.stdout.splitlines() if "iteration:" in l and "residual" in l]
    return {"C": C[: k * k].reshape(k, k).tolist(), "solve_s": solve, "iterations": its,
            "build": "reference CUDA build, stock FP64 PCG one load case at a time, zero guess"}


def elastic256_record():
    """The 256^3 elastic GRF job (50 M DOF, 6 load cases), once: mixed + block + learned guess against the
    plain FP64 PCG (one load case at a time), end to end through the public API, with the device
    time, iterations and tensor error of each, and the block operator's roofline at that size."""
    from chfem_b200 import _native, compute_property
    w = WORKLOADS["elastic256_grf_mixed_block_learned"]
    img = make_image(w, 0)
    wd = tempfile.mkdtemp()
    nf, raw = write_case(wd, w, img)
    kw = dict(mat_props=w["props"], voxel_size=1.0, solver_tolerance=w["tol"], solver_maxiter=w["maxit"])
    compute_property("elasticity", img, precision="mixed", multirhs=True, initial_guess="learned", **kw)  # warm
    t0 = time.perf_counter()
    C = np.array(compute_property("elasticity", img, precision="mixed", multirhs=True, initial_guess="learned", **kw))
    t_fast = time.perf_counter() - t0
    st = _native.solve_stats()
    fast = {"e2e_s": t_fast, "device_solve_s": float(sum(st.solve_seconds[i] for i in range(max(1, st.n_cases)))),
            "iterations": [int(st.iterations[i]) for i in range(max(1, st.n_cases))]}
    lib = _native.chfem()
    lib.chfemB200SetQuiet(1)
    flat = np.ascontiguousarray(img.reshape(-1))
    Cp = np.zeros(36)
    t0 = time.perf_counter()
    lib.chfemB200Run(flat.ctypes.data_as(ctypes.c_void_p), nf.encode(), 6, 0, 1, 0, 0, Cp.ctypes.data_as(ctypes.c_void_p))
    t_plain = time.perf_counter() - t0
    st = _native.solve_stats()
    plain = {"e2e_s": t_plain, "device_solve_s": float(sum(st.solve_seconds[i] for i in range(max(1, st.n_cases)))),
             "iterations": [int(st.iterations[i]) for i in range(max(1, st.n_cases))]}
    Cp = Cp.reshape(6, 6)
    m = Resident(nf, raw, w)
    rl = dominant_kernel_roofline(m, w, True, "elastic256_grf_mixed_block_learned")
    m.close()
    return {"workload": "elastic256_grf_mixed_block_learned", "shape_zyx": list(w["shape"]), "dof": 3 * img.size, "load_cases": 6,
            "mixed_block_learned": fast, "plain_fp64_pcg": plain, "e2e_speedup": t_plain / t_fast,
            "tensor_rel_err_vs_plain_fp64": rel_to_max(C, Cp), "roofline": rl}

if __name__ == "__main__":
    main()
