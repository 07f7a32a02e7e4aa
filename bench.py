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
    "thermal64_spheres_fp64": dict(analysis=0, shape=(64, 64, 64), gen="spheres", vf=0.30, seed=1000,
                                   props={0: 1.0, 255: 10.0}, tol=1e-6, maxit=20000, precision="fp64"),
    "elastic128_grf_mixed_block": dict(analysis=1, shape=(128, 128, 128), gen="grf", corr=6.0, fraction=0.40, seed=2000,
                                       props={0: (1.0, 0.30), 255: (10.0, 0.20)}, tol=1e-6, maxit=20000,
                                       precision="mixed", multirhs=True),
    "thermal64_spheres_fp64_block": dict(analysis=0, shape=(64, 64, 64), gen="spheres", vf=0.30, seed=1000,
                                         props={0: 1.0, 255: 10.0}, tol=1e-6, maxit=20000, precision="fp64",
                                         multirhs=True),
    # Stokes solves run in FP64 in every precision mode (the (P)MINRES recurrence nears breakdown
    # on the indefinite system, where FP32 rounding stalls it)
    "stokes128_grf_fp64": dict(analysis=2, shape=(128, 128, 128), gen="pore", corr=8.0, porosity=0.35, seed=3000,
                               props=None, tol=1e-6, maxit=100000, precision="fp64", solver=1),
    "stokes128_grf_fp64_block": dict(analysis=2, shape=(128, 128, 128), gen="pore", corr=8.0, porosity=0.35, seed=3000,
                                     props=None, tol=1e-6, maxit=100000, precision="fp64", solver=1, multirhs=True),
}
DEFAULT = "elastic128_grf_mixed_block"


def make_image(w, rank):
    from chfem_b200 import synthetic
    seed = w["seed"] + rank
    if w["gen"] == "grf":
        return synthetic.grf(w["shape"], corr=w["corr"], fraction=w["fraction"], seed=seed)
    if w["gen"] == "spheres":
        return synthetic.spheres(w["shape"], vf=w["vf"], seed=seed)
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

    def kernel_time(self, which, reps=20):
        self.c.cudapcgB200TimeKernel.restype = ctypes.c_double
        return self.c.cudapcgB200TimeKernel(which, reps)

    def close(self):
        self.c.cudapcgEnd()
        self.h.hmgEnd()


def e2e_step(img, nf, w):
    """One homogenization through the public API's native entry (compute_property's path)."""
    from chfem_b200 import _native
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


def reference_arm(args, w):
    exe = os.path.join(ROOT, "oracle", "_ref", "chfem_exec_ref")
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "reference CUDA build oracle/_ref/chfem_exec_ref not built"}))
        return
    img = make_image(w, 0)
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
                "config": config_dict(args, w, 1) | {"reference_build": "stock FP64, 16-bit keys, 128 threads/block, sm_100a"},
                "iterations": its,
                "cpu_baseline": {"value": v, "unit": "s", "cores": 0, "kind": "reference",
                                 "sample": "reference CUDA build (its only solver path) on the same B200, full workload"},
                "e2e": {"value": float(np.mean(walls)), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    return "time-to-tol 1e-6 (s): all load cases of the workload, device time, model resident"


def config_dict(args, w, n):
    return {"workload": args.workload, "shape_zyx": list(w["shape"]), "analysis": ["thermal", "elastic", "stokes"][w["analysis"]],
            "load_cases": 6 if w["analysis"] == 1 else 3, "tol": w["tol"], "precision": w["precision"],
            "solver": "PMINRES" if w.get("solver", 0) == 1 else "PCG", "preconditioner": "Jacobi",
            "multirhs": bool(w.get("multirhs", False)),
            "l2": "working set > L2 (vectors of the elastic 128^3 case ~25-50 MB each)", "parallelism": f"samples x{n}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:  # one GPU per process: pin before any CUDA context exists
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = vis.split(",") if vis else [str(i) for i in range(64)]
        os.environ["CUDA_VISIBLE_DEVICES"] = devs[local]
    if args.impl == "reference":
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
    for _ in range(args.warmup):
        model.step(block)
    clocks = Clocks()
    barrier()
    clocks.start()
    t0 = time.perf_counter()
    dev_total, its, launches = 0.0, None, 0
    for _ in range(args.steps):
        d, its, l = model.step(block)
        dev_total += d
        launches += l
    wall = time.perf_counter() - t0
    barrier()
    clk = clocks.stop()
    step_s = allmax(dev_total / args.steps)
    wall_step = allmax(wall / args.steps)
    # dominant kernel, timed live on the library's stream
    peak, peak_kind = load_peaks()
    prec = w["precision"]
    es = 4 if prec == "mixed" else 8
    if w["analysis"] == 2:
        kern_which, kname = 3, "k_fl_apply<MR> (Stokes operator + PMINRES step, one right-hand side)"
        per_unit = 4 * es * 4 + 4 * 2  # per DOF row set, approximate
        units = model.ndof
    else:
        nd = 3 if w["analysis"] == 1 else 1
        tn = 'float' if es == 4 else 'double'
        if block:
            nr = 6 if nd == 3 else 3
            kern_which, kname = 5, f"k_blk_apply<{nd},{tn},{nr}> (block operator + directions + dots, {nr} load cases)"
            per_unit = nr * 4 * nd * es + 2  # per load case s, d_old in; d_new, q out; one 16-bit key
        else:
            kern_which, kname = 1, f"k_te_apply<{nd},{tn},TE_PCG> (operator + direction + dot)"
            per_unit = 4 * nd * es + 2  # s, d_old in; d_new, q out (nd comps); 16-bit key
        units = model.N
    kt = model.kernel_time(kern_which, reps=30)
    achieved = per_unit * units / kt / 1e9 if kt > 0 else None
    fl_unit = (1152 if w["analysis"] == 1 else 80) * ((6 if w["analysis"] == 1 else 3) if block else 1)
    flops = fl_unit * units / kt / 1e12 if (kt > 0 and w["analysis"] != 2) else None
    traffic = profiled_traffic(args.workload)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "kernel": kname, "kernel_ms": kt * 1e3, "bytes_per_unit": per_unit, "units_per_launch": units,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                "fp_tflops_achieved": flops}
    total_its = sum(its)
    dof_its = model.ndof * total_its / (dev_total / args.steps)
    # e2e through the public API (host image in, tensor out)
    e2e_times = []
    C = None
    st = None
    breakdown = None
    for k in range(2):
        t, C, st = e2e_step(img, nf, w)
        if not e2e_times or t < min(e2e_times):
            ncs = max(1, st.n_cases)
            breakdown = {"model_build_and_upload_s": t - st.total_seconds, "rhs_assembly_s": st.rhs_seconds,
                         "solve_device_s": float(sum(st.solve_seconds[i] for i in range(ncs))),
                         "tensor_update_s": st.update_seconds, "solver_call_total_s": st.total_seconds}
        e2e_times.append(t)
    e2e = allmax(min(e2e_times))
    ncase = 6 if w["analysis"] == 1 else 3
    maps = 2 * model.N if w["analysis"] != 2 else 9 * model.N  # node keys, or the Stokes DOF maps
    if block:  # right-hand sides and tensor volume terms stay on the device
        ns = 6 if w["analysis"] == 1 else 3
        h2d = int(img.size + maps)
        d2h = int(ncase * ns * 8)
    else:
        h2d = int(img.size + maps + ncase * model.ndof * 8)
        d2h = int(ncase * model.ndof * 8)
    model.close()
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        its64 = sum(fp64["iterations"]) if fp64 else total_its
        cpu = cpu_baseline(wd, w, img, its64)
    if rank == 0:
        line = {"metric": metric_name(w), "value": step_s, "unit": "s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64" if prec == "mixed" else "f64", "data": "synthetic",
                "config": config_dict(args, w, world),
                "iterations": its, "dof_iterations_per_s": dof_its, "wall_s_per_step": wall_step,
                "plain_fp64_pcg": fp64, "speedup_vs_plain_fp64": (fp64["time_s"] / step_s) if fp64 else None,
                "tensor_diag": [float(C[i, i]) for i in range(C.shape[0])] if C is not None else None,
                "roofline": roofline, "clocks": clk, "gpu_launches": int(launches),
                "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "path": "chfemB200Run (compute_property's native entry): image in host memory -> tensor",
                        "breakdown": breakdown},
                "cpu_baseline": cpu, "samples_per_s": world / step_s}
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
