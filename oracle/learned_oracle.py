"""CPU oracle of the learned initial guess's network (test infrastructure only).

A NumPy, FP64 restatement of the periodic 3D U-Net of chfem_b200/learned.py -- the same layer
list, parameter layout and operations (periodic 3x3x3 / 1x1x1 cross-correlation, ReLU, 2x2x2
average pooling, nearest 2x upsampling, channel concatenation), with its backward pass written
out by hand.  The tests pin it by finite differences and then check the CUDA kernels' forward
outputs and parameter gradients against it.  Nothing in the product imports this file.
"""
import numpy as np

CH = (16, 32, 48, 64)
IN_CH = 2
OUT_CH = 18
LAYERS = [("enc0", CH[0], IN_CH, 3), ("enc1", CH[1], CH[0], 3), ("enc2", CH[2], CH[1], 3), ("enc3", CH[3], CH[2], 3),
          ("dec2", CH[2], CH[3] + CH[2], 3), ("dec1", CH[1], CH[2] + CH[1], 3), ("dec0", CH[0], CH[1] + CH[0], 3),
          ("head", OUT_CH, CH[0], 1)]


def offsets():
    out, n = {}, 0
    for name, co, ci, k in LAYERS:
        out[name] = (n, n + co * ci * k ** 3, co, ci, k)
        n += co * ci * k ** 3 + co
    return out, n


def _taps(k):
    r = range(-(k // 2), k // 2 + 1)
    return [(dz, dy, dx) for dz in r for dy in r for dx in r]


def conv(x, w, b, k):
    """x [C, D, H, W] -> out[co] = b[co] + sum_ci sum_o w[co, ci, o] x[ci][p + d_o] (periodic)."""
    co_n, ci_n = w.shape[0], w.shape[1]
    out = np.zeros((co_n,) + x.shape[1:])
    for o, (dz, dy, dx) in enumerate(_taps(k)):
        xs = np.roll(x, shift=(-dz, -dy, -dx), axis=(1, 2, 3))
        out += np.einsum("oc,cdhw->odhw", w[:, :, o], xs)
    return out + b[:, None, None, None]


def conv_bwd(x, w, k, g):
    """(dL/dx, dL/dw, dL/db) of conv given g = dL/d(out)."""
    gx = np.zeros_like(x)
    gw = np.zeros_like(w)
    for o, (dz, dy, dx) in enumerate(_taps(k)):
        xs = np.roll(x, shift=(-dz, -dy, -dx), axis=(1, 2, 3))
        gw[:, :, o] = np.einsum("odhw,cdhw->oc", g, xs)
        gx += np.roll(np.einsum("oc,odhw->cdhw", w[:, :, o], g), shift=(dz, dy, dx), axis=(1, 2, 3))
    return gx, gw, g.sum(axis=(1, 2, 3))


def pool(x):
    C, D, H, W = x.shape
    return x.reshape(C, D // 2, 2, H // 2, 2, W // 2, 2).mean(axis=(2, 4, 6))


def pool_bwd(g):
    return np.repeat(np.repeat(np.repeat(g, 2, 1), 2, 2), 2, 3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 1), 2, 2), 2, 3)


def up_bwd(g):
    C, D, H, W = g.shape
    return g.reshape(C, D // 2, 2, H // 2, 2, W // 2, 2).sum(axis=(2, 4, 6))


class UNet:
    def __init__(self, params):
        self.off, n = offsets()
        assert params.size == n
        self.p = np.asarray(params, np.float64)

    def wb(self, name):
        w0, b0, co, ci, k = self.off[name]
        return self.p[w0:b0].reshape(co, ci, k ** 3), self.p[b0:b0 + co], k

    def forward(self, feat):
        """feat [2, D, H, W] -> [18, D, H, W]; keeps what backward needs."""
        relu = lambda v: np.maximum(v, 0.0)
        c = {}
        c["in"] = feat
        c["x0"] = relu(conv(feat, *self.wb("enc0")))
        c["p1"] = pool(c["x0"])
        c["x1"] = relu(conv(c["p1"], *self.wb("enc1")))
        c["p2"] = pool(c["x1"])
        c["x2"] = relu(conv(c["p2"], *self.wb("enc2")))
        c["p3"] = pool(c["x2"])
        c["x3"] = relu(conv(c["p3"], *self.wb("enc3")))
        c["cat2"] = np.concatenate([up(c["x3"]), c["x2"]])
        c["d2"] = relu(conv(c["cat2"], *self.wb("dec2")))
        c["cat1"] = np.concatenate([up(c["d2"]), c["x1"]])
        c["d1"] = relu(conv(c["cat1"], *self.wb("dec1")))
        c["cat0"] = np.concatenate([up(c["d1"]), c["x0"]])
        c["d0"] = relu(conv(c["cat0"], *self.wb("dec0")))
        c["out"] = conv(c["d0"], *self.wb("head"))
        self.c = c
        return c["out"]

    def backward(self, g_out):
        """Flat parameter gradient given dL/d(out)."""
        c = self.c
        grad = np.zeros_like(self.p)

        def put(name, gw, gb):
            w0, b0, co, ci, k = self.off[name]
            grad[w0:b0] += gw.reshape(-1)
            grad[b0:b0 + co] += gb

        def cb(name, x, g):
            w, _, k = self.wb(name)
            gx, gw, gb = conv_bwd(x, w, k, g)
            put(name, gw, gb)
            return gx

        g = cb("head", c["d0"], g_out) * (c["d0"] > 0)
        g_cat0 = cb("dec0", c["cat0"], g)
        g = up_bwd(g_cat0[:CH[1]]) * (c["d1"] > 0)
        g_cat1 = cb("dec1", c["cat1"], g)
        g = up_bwd(g_cat1[:CH[2]]) * (c["d2"] > 0)
        g_cat2 = cb("dec2", c["cat2"], g)
        g = up_bwd(g_cat2[:CH[3]]) * (c["x3"] > 0)
        g_p3 = cb("enc3", c["p3"], g)
        g = (g_cat2[CH[3]:] + pool_bwd(g_p3)) * (c["x2"] > 0)
        g_p2 = cb("enc2", c["p2"], g)
        g = (g_cat1[CH[2]:] + pool_bwd(g_p2)) * (c["x1"] > 0)
        g_p1 = cb("enc1", c["p1"], g)
        g = (g_cat0[CH[1]:] + pool_bwd(g_p1)) * (c["x0"] > 0)
        cb("enc0", c["in"], g)
        return grad
