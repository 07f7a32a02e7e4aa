"""The CPU oracle of the learned guess's network, pinned by finite differences (CPU only)."""
import os
import sys

import numpy as np

from tests import helpers as H

sys.path.insert(0, os.path.join(H.ROOT, "oracle"))
import learned_oracle as LO  # noqa: E402


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    off, n = LO.offsets()
    p = rng.standard_normal(n) * 0.2
    feat = rng.standard_normal((2, 8, 8, 8))
    R = rng.standard_normal((LO.OUT_CH, 8, 8, 8))
    net = LO.UNet(p)
    net.forward(feat)
    g = net.backward(R)
    loss = lambda q: float((LO.UNet(q).forward(feat) * R).sum())
    h = 1e-6
    idx = list(rng.choice(n, 40, replace=False))
    for name in ("enc0", "dec2", "head"):  # a weight and a bias of a few layers for sure
        w0, b0, co, ci, k = off[name]
        idx += [w0 + 3, b0]
    for i in idx:
        e = np.zeros(n)
        e[i] = h
        fd = (loss(p + e) - loss(p - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_oracle_building_blocks_are_adjoint():
    """<conv(x), y> = <x, conv^T(y)>, and the pool / upsample pairs, on random periodic fields."""
    rng = np.random.default_rng(4)
    for k in (1, 3):
        x = rng.standard_normal((3, 4, 6, 8))
        w = rng.standard_normal((5, 3, k ** 3))
        y = rng.standard_normal((5, 4, 6, 8))
        out = LO.conv(x, w, np.zeros(5), k)
        gx, gw, _ = LO.conv_bwd(x, w, k, y)
        assert np.isclose((out * y).sum(), (x * gx).sum())
    x = rng.standard_normal((2, 4, 4, 8))
    y = rng.standard_normal((2, 2, 2, 4))
    assert np.isclose((LO.pool(x) * y).sum(), (x * LO.pool_bwd(y)).sum())
    assert np.isclose((LO.up(y) * x).sum(), (y * LO.up_bwd(x)).sum())
