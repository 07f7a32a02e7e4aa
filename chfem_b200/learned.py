"""Learned initial guess for elastic homogenization.

A small periodic 3D U-Net maps a voxel image's material fields (log stiffness ratio, Poisson
ratio) to the periodic fluctuation of the solution of all six elastic load cases; the
macroscopic ramp of each load case is added analytically, and the result is the initial guess
of the PCG solve.  PCG still runs to the requested tolerance (relative to the zero-guess
residual, as in the reference), so the effective tensor is unchanged -- the guess only removes
iterations.  It stands in for the reference's recursive coarse-grid initial-guess search
(chfem/src/femhmg/femhmg.c:561-846), which stays available as the fallback (-r).

Every operation of the network, forward and backward, is a hand-written CUDA kernel of
libcudapcg_b200.so (chfem_b200/csrc/learned.cu); PyTorch only holds the device buffers and the
stream.  Layout: tensors [N][C][L][Cc][R] in chfem's internal node order (row fastest), the
voxel image mapped as img[z][y][x] -> [z][x][y].
"""
import ctypes
import math
import os
import struct

import numpy as np

from . import _native

CH = (16, 32, 48, 64)
IN_CH = 2
OUT_CH = 18  # 6 load cases x 3 displacement components
# layers: name -> (cout, cin, ksize)
LAYERS = [("enc0", CH[0], IN_CH, 3), ("enc1", CH[1], CH[0], 3), ("enc2", CH[2], CH[1], 3), ("enc3", CH[3], CH[2], 3),
          ("dec2", CH[2], CH[3] + CH[2], 3), ("dec1", CH[1], CH[2] + CH[1], 3), ("dec0", CH[0], CH[1] + CH[0], 3),
          ("head", OUT_CH, CH[0], 1)]
CASE_AXIS = (0, 1, 2, 1, 2, 1)  # load cases X Y Z YZ XZ XY: axis of the macroscopic jump
CASE_COMP = (0, 1, 2, 2, 0, 0)  # and the displaced component
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "elastic_unet.bin")
E_SCALE = math.log(50.0)


def _lib():
    lib = _native.cudapcg()
    if not getattr(lib, "_nn_typed", False):
        c = ctypes
        P, L, I, F = c.c_void_p, c.c_long, c.c_int, c.c_float
        lib.chfemB200NnLastError.restype = c.c_char_p
        lib.chfemB200NnConv3d.argtypes = [P, L, I, I, I, I, I, P, P, I, I, I, I, P, L, P]
        lib.chfemB200NnConv3dBackwardData.argtypes = [P, L, I, I, I, I, I, P, I, I, P, I, P, L, P]
        lib.chfemB200NnConv3dBackwardWeight.argtypes = [P, L, I, I, I, I, I, P, L, I, I, P, P, P]
        lib.chfemB200NnReluBackward.argtypes = [P, L, P, L, L, I, P]
        lib.chfemB200NnPool2.argtypes = [P, L, I, I, I, I, I, P, L, P]
        lib.chfemB200NnPool2Backward.argtypes = [P, L, I, I, I, I, I, P, L, I, P]
        lib.chfemB200NnUpsample2.argtypes = [P, L, I, I, I, I, I, P, L, P]
        lib.chfemB200NnUpsample2Backward.argtypes = [P, L, I, I, I, I, I, P, L, P]
        lib.chfemB200NnMse.argtypes = [P, P, L, P, P, P]
        lib.chfemB200NnAdam.argtypes = [P, P, P, P, L, F, F, F, F, I, P]
        lib.chfemB200NnFeatures.argtypes = [P, L, L, P, I, P, L, I, P]
        lib._nn_typed = True
    return lib


def _ok(rc):
    if not rc:
        raise RuntimeError(_lib().chfemB200NnLastError().decode())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t, offset=0):
    return ctypes.c_void_p(t.data_ptr() + 4 * offset)


class Net:
    """The U-Net: parameters, gradients and Adam moments as flat FP32 device tensors."""

    def __init__(self, seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.device = device
        self.offsets = {}
        n = 0
        for name, co, ci, k in LAYERS:
            self.offsets[name] = (n, n + co * ci * k ** 3, co, ci, k)
            n += co * ci * k ** 3 + co
        self.nparams = n
        rng = np.random.default_rng(seed)
        p = np.zeros(n, np.float32)
        for name, co, ci, k in LAYERS:
            w0, b0, _, _, _ = self.offsets[name]
            std = math.sqrt(2.0 / (ci * k ** 3)) if name != "head" else 1e-3
            p[w0:b0] = rng.standard_normal(co * ci * k ** 3).astype(np.float32) * std
        self.p = torch.tensor(p, device=device)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.wt = torch.zeros(max(co * ci * k ** 3 for _, co, ci, k in LAYERS), device=device)
        self.step_count = 0
        self.acts = None

    # -- parameters ------------------------------------------------------------------
    def w(self, name, grad=False):
        w0, b0, co, ci, k = self.offsets[name]
        return ptr(self.g if grad else self.p, w0), ptr(self.g if grad else self.p, b0)

    def save(self, path):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "wb") as f:
            f.write(b"CHFEMNN1")
            f.write(struct.pack("<i", self.nparams))
            f.write(self.p.detach().cpu().numpy().astype("<f4").tobytes())

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS, device="cuda"):
        import torch
        with open(path, "rb") as f:
            if f.read(8) != b"CHFEMNN1":
                raise ValueError(f"{path}: not a chfem_b200 network file")
            (n,) = struct.unpack("<i", f.read(4))
            p = np.frombuffer(f.read(4 * n), dtype="<f4")
        net = cls(device=device)
        if n != net.nparams:
            raise ValueError(f"{path}: {n} parameters, the network has {net.nparams}")
        net.p.copy_(torch.tensor(p, device=device))
        return net

    # -- forward / backward ------------------------------------------------------------
    def _buffers(self, N, D, H, W):
        key = (N, D, H, W)
        if self.acts is not None and self.acts["key"] == key:
            return self.acts
        t = self.torch
        z = lambda c, s: t.zeros((N, c) + s, device=self.device, dtype=t.float32)
        s0, s1, s2, s3 = (D, H, W), (D // 2, H // 2, W // 2), (D // 4, H // 4, W // 4), (D // 8, H // 8, W // 8)
        a = dict(key=key, s=(s0, s1, s2, s3))
        a["cat0"] = z(CH[1] + CH[0], s0)   # [up(d1) | x0]
        a["cat1"] = z(CH[2] + CH[1], s1)   # [up(d2) | x1]
        a["cat2"] = z(CH[3] + CH[2], s2)   # [up(x3) | x2]
        a["p1"], a["p2"], a["p3"] = z(CH[0], s1), z(CH[1], s2), z(CH[2], s3)
        a["x3"] = z(CH[3], s3)
        a["d2"], a["d1"], a["d0"] = z(CH[2], s2), z(CH[1], s1), z(CH[0], s0)
        a["out"] = z(OUT_CH, s0)
        self.acts = a
        return a

    def _grad_buffers(self, a):
        if "g_cat0" in a:
            return
        for k in ("cat0", "cat1", "cat2", "p1", "p2", "p3", "x3", "d2", "d1", "d0", "out"):
            a["g_" + k] = self.torch.zeros_like(a[k])

    def forward(self, feat):
        """feat: [N, 2, D, H, W] float32 CUDA tensor (D, H, W divisible by 8) -> [N, 18, D, H, W]."""
        lib, st = _lib(), _stream()
        N, _, D, H, W = feat.shape
        if D % 8 or H % 8 or W % 8:
            raise ValueError("the network needs every axis divisible by 8")
        a = self._buffers(N, D, H, W)
        (s0, s1, s2, s3) = a["s"]
        S = lambda s: s[0] * s[1] * s[2]
        ns = lambda name: a[name].shape[1] * S(a[name].shape[2:])
        def conv(name, src, src_off, src_ns, C_in, s, dst, dst_off, dst_ns, relu):
            wp, bp = self.w(name)
            _, _, co, ci, k = self.offsets[name]
            assert ci == C_in
            _ok(lib.chfemB200NnConv3d(ptr(src, src_off), src_ns, N, ci, *s, wp, bp, co, k, relu, 0, ptr(dst, dst_off), dst_ns, st))
        # encoder; the skip features live in the upper channel slices of the concatenation buffers
        conv("enc0", feat, 0, IN_CH * S(s0), IN_CH, s0, a["cat0"], CH[1] * S(s0), ns("cat0"), 1)
        _ok(lib.chfemB200NnPool2(ptr(a["cat0"], CH[1] * S(s0)), ns("cat0"), N, CH[0], *s0, ptr(a["p1"]), ns("p1"), st))
        conv("enc1", a["p1"], 0, ns("p1"), CH[0], s1, a["cat1"], CH[2] * S(s1), ns("cat1"), 1)
        _ok(lib.chfemB200NnPool2(ptr(a["cat1"], CH[2] * S(s1)), ns("cat1"), N, CH[1], *s1, ptr(a["p2"]), ns("p2"), st))
        conv("enc2", a["p2"], 0, ns("p2"), CH[1], s2, a["cat2"], CH[3] * S(s2), ns("cat2"), 1)
        _ok(lib.chfemB200NnPool2(ptr(a["cat2"], CH[3] * S(s2)), ns("cat2"), N, CH[2], *s2, ptr(a["p3"]), ns("p3"), st))
        conv("enc3", a["p3"], 0, ns("p3"), CH[2], s3, a["x3"], 0, ns("x3"), 1)
        # decoder
        _ok(lib.chfemB200NnUpsample2(ptr(a["x3"]), ns("x3"), N, CH[3], *s3, ptr(a["cat2"]), ns("cat2"), st))
        conv("dec2", a["cat2"], 0, ns("cat2"), CH[3] + CH[2], s2, a["d2"], 0, ns("d2"), 1)
        _ok(lib.chfemB200NnUpsample2(ptr(a["d2"]), ns("d2"), N, CH[2], *s2, ptr(a["cat1"]), ns("cat1"), st))
        conv("dec1", a["cat1"], 0, ns("cat1"), CH[2] + CH[1], s1, a["d1"], 0, ns("d1"), 1)
        _ok(lib.chfemB200NnUpsample2(ptr(a["d1"]), ns("d1"), N, CH[1], *s1, ptr(a["cat0"]), ns("cat0"), st))
        conv("dec0", a["cat0"], 0, ns("cat0"), CH[1] + CH[0], s0, a["d0"], 0, ns("d0"), 1)
        conv("head", a["d0"], 0, ns("d0"), CH[0], s0, a["out"], 0, ns("out"), 0)
        self.feat = feat
        return a["out"]

    def backward(self, g_out):
        """Gradient of the loss w.r.t. the parameters (into self.g) given dL/d(out)."""
        lib, st = _lib(), _stream()
        a = self.acts
        self._grad_buffers(a)
        N = g_out.shape[0]
        (s0, s1, s2, s3) = a["s"]
        S = lambda s: s[0] * s[1] * s[2]
        ns = lambda name: a[name].shape[1] * S(a[name].shape[2:])
        self.g.zero_()

        def conv_bwd(name, src, src_off, src_ns, s, g, g_off, g_ns, gin, gin_off, gin_ns):
            wp, _ = self.w(name)
            gw, gb = self.w(name, grad=True)
            _, _, co, ci, k = self.offsets[name]
            _ok(lib.chfemB200NnConv3dBackwardWeight(ptr(src, src_off), src_ns, N, ci, *s, ptr(g, g_off), g_ns, co, k, gw, gb, st))
            if gin is not None:
                _ok(lib.chfemB200NnConv3dBackwardData(ptr(g, g_off), g_ns, N, co, *s, wp, ci, k, ptr(self.wt), 0,
                                                      ptr(gin, gin_off), gin_ns, st))

        def relu_bwd(y, y_off, y_ns, g, g_off, g_ns, per):
            _ok(lib.chfemB200NnReluBackward(ptr(y, y_off), y_ns, ptr(g, g_off), g_ns, per, N, st))

        conv_bwd("head", a["d0"], 0, ns("d0"), s0, g_out, 0, OUT_CH * S(s0), a["g_d0"], 0, ns("d0"))
        relu_bwd(a["d0"], 0, ns("d0"), a["g_d0"], 0, ns("d0"), CH[0] * S(s0))
        conv_bwd("dec0", a["cat0"], 0, ns("cat0"), s0, a["g_d0"], 0, ns("d0"), a["g_cat0"], 0, ns("cat0"))
        _ok(lib.chfemB200NnUpsample2Backward(ptr(a["g_cat0"]), ns("cat0"), N, CH[1], *s1, ptr(a["g_d1"]), ns("d1"), st))
        relu_bwd(a["d1"], 0, ns("d1"), a["g_d1"], 0, ns("d1"), CH[1] * S(s1))
        conv_bwd("dec1", a["cat1"], 0, ns("cat1"), s1, a["g_d1"], 0, ns("d1"), a["g_cat1"], 0, ns("cat1"))
        _ok(lib.chfemB200NnUpsample2Backward(ptr(a["g_cat1"]), ns("cat1"), N, CH[2], *s2, ptr(a["g_d2"]), ns("d2"), st))
        relu_bwd(a["d2"], 0, ns("d2"), a["g_d2"], 0, ns("d2"), CH[2] * S(s2))
        conv_bwd("dec2", a["cat2"], 0, ns("cat2"), s2, a["g_d2"], 0, ns("d2"), a["g_cat2"], 0, ns("cat2"))
        _ok(lib.chfemB200NnUpsample2Backward(ptr(a["g_cat2"]), ns("cat2"), N, CH[3], *s3, ptr(a["g_x3"]), ns("x3"), st))
        relu_bwd(a["x3"], 0, ns("x3"), a["g_x3"], 0, ns("x3"), CH[3] * S(s3))
        conv_bwd("enc3", a["p3"], 0, ns("p3"), s3, a["g_x3"], 0, ns("x3"), a["g_p3"], 0, ns("p3"))
        # x2 gradient = skip part of g_cat2 + pooled path
        off2 = CH[3] * S(s2)
        _ok(lib.chfemB200NnPool2Backward(ptr(a["g_p3"]), ns("p3"), N, CH[2], *s2, ptr(a["g_cat2"], off2), ns("cat2"), 1, st))
        relu_bwd(a["cat2"], off2, ns("cat2"), a["g_cat2"], off2, ns("cat2"), CH[2] * S(s2))
        conv_bwd("enc2", a["p2"], 0, ns("p2"), s2, a["g_cat2"], off2, ns("cat2"), a["g_p2"], 0, ns("p2"))
        off1 = CH[2] * S(s1)
        _ok(lib.chfemB200NnPool2Backward(ptr(a["g_p2"]), ns("p2"), N, CH[1], *s1, ptr(a["g_cat1"], off1), ns("cat1"), 1, st))
        relu_bwd(a["cat1"], off1, ns("cat1"), a["g_cat1"], off1, ns("cat1"), CH[1] * S(s1))
        conv_bwd("enc1", a["p1"], 0, ns("p1"), s1, a["g_cat1"], off1, ns("cat1"), a["g_p1"], 0, ns("p1"))
        off0 = CH[1] * S(s0)
        _ok(lib.chfemB200NnPool2Backward(ptr(a["g_p1"]), ns("p1"), N, CH[0], *s0, ptr(a["g_cat0"], off0), ns("cat0"), 1, st))
        relu_bwd(a["cat0"], off0, ns("cat0"), a["g_cat0"], off0, ns("cat0"), CH[0] * S(s0))
        conv_bwd("enc0", self.feat, 0, IN_CH * S(s0), s0, a["g_cat0"], off0, ns("cat0"), None, 0, 0)

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        _ok(_lib().chfemB200NnAdam(ptr(self.p), ptr(self.g), ptr(self.m), ptr(self.v), self.nparams, lr, b1, b2, eps,
                                   self.step_count, _stream()))

    def mse(self, pred, target, grad):
        """Mean squared error (a float) and its gradient into grad (may be None)."""
        t = self.torch
        loss = t.zeros(1, dtype=t.float64, device=self.device)
        _ok(_lib().chfemB200NnMse(ptr(pred), ptr(target), pred.numel(), ptr(grad) if grad is not None else None,
                                  ctypes.c_void_p(loss.data_ptr()), _stream()))
        return float(loss.item())


# ---------------------------------------------------------------------------------------
# Problem <-> network tensors
def features(images, props, device="cuda"):
    """[N, 2, L, C, R] material features of uint8 (z, y, x) images with one {colour: (E, nu)} dict
    each: log(E / E_min) / log(50) and (nu - 0.25) * 4."""
    import torch
    imgs = [np.ascontiguousarray(np.asarray(im, np.uint8).transpose(0, 2, 1)) for im in images]
    N = len(imgs)
    shape = imgs[0].shape
    table = np.zeros((N, 256, 2), np.float32)
    for n, p in enumerate(props):
        emin = min(v[0] for v in p.values())
        for c, (E, nu) in p.items():
            table[n, int(c)] = (math.log(E / emin) / E_SCALE, (nu - 0.25) * 4.0)
    img_t = torch.tensor(np.stack(imgs), device=device)
    out = torch.zeros((N, 2) + shape, device=device, dtype=torch.float32)
    S = int(np.prod(shape))
    tab = torch.tensor(table, device=device)
    for n in range(N):
        _ok(_lib().chfemB200NnFeatures(ctypes.c_void_p(img_t.data_ptr() + n * S), S, S, ptr(tab[n]), 2,
                                       ptr(out, n * 2 * S), 2 * S, 1, _stream()))
    return out


def ramp(shape_lcr, case):
    """The macroscopic part of load case `case` in chfem's solution vector (the homogeneous-medium
    solution up to a constant): component CASE_COMP[case] equals col (x), (R - row) mod R (y) or
    (L - layer) mod L (z) on the nodes, array [L][C][R]."""
    L, C, R = shape_lcr
    axis = CASE_AXIS[case]
    if axis == 0:
        v = np.broadcast_to(np.arange(C, dtype=np.float64)[None, :, None], (L, C, R))
    elif axis == 1:
        v = np.broadcast_to(((R - np.arange(R)) % R).astype(np.float64)[None, None, :], (L, C, R))
    else:
        v = np.broadcast_to(((L - np.arange(L)) % L).astype(np.float64)[:, None, None], (L, C, R))
    return v


def fluctuation(xs, shape_lcr):
    """[18, L, C, R] float32 periodic part (zero-mean per channel) of the six solution vectors
    xs[k] (chfem layout: node-major, 3 components)."""
    L, C, R = shape_lcr
    out = np.zeros((OUT_CH, L, C, R), np.float32)
    for k in range(6):
        x = np.asarray(xs[k], np.float64).reshape(L, C, R, 3)
        for comp in range(3):
            f = x[..., comp] - (ramp(shape_lcr, k) if comp == CASE_COMP[k] else 0.0)
            out[3 * k + comp] = f - f.mean()
    return out


_NET = {}


def default_net():
    """The committed trained network (loaded once)."""
    if "net" not in _NET:
        _NET["net"] = Net.load(DEFAULT_WEIGHTS)
    return _NET["net"]


def device_guesses(net, img, props):
    """The six initial-guess vectors for one image as FP64 CUDA tensors (network forward pass
    and the ramps assembled on the device; nothing crosses to the host)."""
    import torch
    lib = _lib()
    feat = features([img], [props])
    out = net.forward(feat)
    L, C, R = out.shape[2:]
    xs = [torch.empty(3 * L * C * R, dtype=torch.float64, device="cuda") for _ in range(6)]
    P = ctypes.c_void_p * 6
    lib.chfemB200NnAssembleGuess.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p]
    _ok(lib.chfemB200NnAssembleGuess(ptr(out), L, C, R, P(*[x.data_ptr() for x in xs]), _stream()))
    return xs


def initial_guesses(net, img, props, device="cuda"):
    """The six initial-guess vectors (chfem layout, float64 host arrays) for one image."""
    feat = features([img], [props], device)
    out = net.forward(feat)[0].detach().cpu().numpy().astype(np.float64)
    L, C, R = out.shape[1:]
    xs = []
    for k in range(6):
        x = np.zeros((L, C, R, 3))
        for comp in range(3):
            x[..., comp] = out[3 * k + comp] + (ramp((L, C, R), k) if comp == CASE_COMP[k] else 0.0)
        xs.append(np.ascontiguousarray(x.reshape(-1)))
    return xs


# ---------------------------------------------------------------------------------------
# Reference solutions with the native solver (all six load cases as one block)
def solve_elastic(img, props, tol=1e-6, maxit=20000, precision="mixed", x0=None, want_x=True):
    """(C 6x6, iterations[6], list of 6 solution vectors or None) for one image via the host
    layer and cudapcgB200SolveLoadCases; x0: optional six initial-guess vectors."""
    import tempfile
    from .io import export_for_chfem
    from ._native import setup_cudapcg_model
    h, c = _native.chfem(), _native.cudapcg()
    h.chfemB200SetQuiet(1)
    with tempfile.TemporaryDirectory() as d:
        prefix = os.path.join(d, "s")
        export_for_chfem(prefix + ".raw", img, 1, mat_props=props, voxel_size=1.0, solver_tolerance=tol, solver_maxiter=maxit,
                         export_raw=False, export_nf=True)
        flat = np.ascontiguousarray(np.asarray(img, np.uint8).reshape(-1))
        if not h.hmgInit((prefix + ".nf").encode(), None, None, flat.ctypes.data_as(ctypes.c_void_p)):
            raise RuntimeError(h.chfemB200LastError().decode())
    info = (ctypes.c_uint * 9)()
    h.chfemB200ModelInfo(info)

    def arr(wh, t):
        n = h.chfemB200ModelArraySize(wh)
        x = np.zeros(n // np.dtype(t).itemsize, dtype=t)
        if n:
            h.chfemB200CopyModelArray(wh, x.ctypes.data_as(ctypes.c_void_p), n)
        return x
    a = dict(nx=info[0], ny=info[1], nz=info[2], N=info[3], ndof=info[4], nV=info[5], nB=info[6], nkeys=info[7],
             analysis=info[8], keys=arr(0, np.uint16), dof_of_node=arr(1, np.uint32), node_of_dof=arr(2, np.uint32),
             border=arr(3, np.uint8), lcl=arr(4, np.float64))
    CB = arr(7, np.float64)
    setup_cudapcg_model(c, a)
    c.cudapcgSetSolver(0)
    c.cudapcgSetPreconditioner(1)
    c.cudapcgSetNumTol(ctypes.c_double(tol))
    c.cudapcgSetMaxIterations(maxit)
    c.cudapcgB200SetPrecision(1 if precision == "mixed" else 0)
    if not c.cudapcgAllocateArrays():
        raise RuntimeError(c.cudapcgB200LastError().decode())
    nx, ny, nz = info[0], info[1], info[2]
    axis = (ctypes.c_int * 6)(*CASE_AXIS)
    comp = (ctypes.c_int * 6)(*CASE_COMP)
    jump = (ctypes.c_double * 6)(*[float((nx, ny, nz)[ax]) for ax in CASE_AXIS])
    ndof = info[4]
    xs = [np.zeros(ndof) for _ in range(6)] if want_x else None
    P = ctypes.c_void_p * 6
    px = P(*[x.ctypes.data for x in xs]) if want_x else None
    x0s = [np.ascontiguousarray(v, dtype=np.float64) for v in x0] if x0 is not None else None
    px0 = P(*[v.ctypes.data for v in x0s]) if x0s is not None else None
    vol = np.zeros(36)
    its = (ctypes.c_uint * 6)()
    res = (ctypes.c_double * 6)()
    rc = c.cudapcgB200SolveLoadCases(6, axis, comp, jump, CB.ctypes.data_as(ctypes.c_void_p), 6, px0, 0,
                                     vol.ctypes.data_as(ctypes.c_void_p), px, its, res)
    err = c.cudapcgB200LastError()
    if not rc and err:
        raise RuntimeError(err.decode())
    st = _native.CudapcgStats()
    c.cudapcgB200GetStats(ctypes.byref(st))
    C = np.zeros((6, 6))
    for k in range(6):
        C[:, k] = vol[6 * k:6 * k + 6]
    C = h_tensor_from_volume(h, C)
    c.cudapcgEnd()
    h.hmgEnd()
    return C, list(its), xs, st.solve_seconds + st.setup_seconds


def h_tensor_from_volume(h, vol_cols):
    """Effective stiffness from the device volume terms: the host layer adds the face terms."""
    C = np.zeros((6, 6))
    out = np.zeros(36)
    for k in range(6):
        h.chfemB200UpdateCFromVolume(k, np.ascontiguousarray(vol_cols[:, k]).ctypes.data_as(ctypes.c_void_p),
                                     out.ctypes.data_as(ctypes.c_void_p))
    return out.reshape(6, 6)
