"""The learned initial guess on the GPU: its hand-written CUDA forward and backward passes
against the CPU oracle (oracle/learned_oracle.py, pinned by finite differences), and what the
trained network gains over the zero guess.

Bars: forward output within 1e-4 and parameter gradients within 1e-3 of the oracle's, relative
to the largest entry (FP32 kernels against the FP64 oracle); with the guess the elastic tensor
equals the zero-guess tensor to the FP64 solver bar (1e-6) in fewer iterations.
"""
import os
import sys

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(H.ROOT, "oracle"))


def test_network_forward_and_gradients_match_oracle():
    import torch
    import learned_oracle as LO
    from chfem_b200 import learned as L
    rng = np.random.default_rng(0)
    net = L.Net(seed=1)
    p = net.p.cpu().numpy().astype(np.float64)
    p[:] = rng.standard_normal(p.size) * 0.15
    net.p.copy_(torch.tensor(p, dtype=torch.float32))
    N, D, Hh, W = 2, 8, 16, 24
    feat = rng.standard_normal((N, 2, D, Hh, W))
    gout = rng.standard_normal((N, L.OUT_CH, D, Hh, W))
    out = net.forward(torch.tensor(feat, dtype=torch.float32, device="cuda")).cpu().numpy()
    net.backward(torch.tensor(gout, dtype=torch.float32, device="cuda"))
    torch.cuda.synchronize()
    g = net.g.cpu().numpy().astype(np.float64)
    gref = np.zeros_like(p)
    pf = net.p.cpu().numpy().astype(np.float64)  # the FP32 parameters the kernels used
    for n in range(N):
        o = LO.UNet(pf)
        ref = o.forward(feat[n])
        assert H.rel_to_max(out[n], ref) < 1e-4
        gref += o.backward(gout[n])
    assert H.rel_to_max(g, gref) < 1e-3
    # per layer too, so a small layer's error is not hidden by a large one
    off, _ = LO.offsets()
    for name, (w0, b0, co, ci, k) in off.items():
        assert H.rel_to_max(g[w0:b0], gref[w0:b0]) < 1e-3, name
        assert H.rel_to_max(g[b0:b0 + co], gref[b0:b0 + co]) < 1e-3, name


def test_adam_and_mse_kernels():
    import torch
    from chfem_b200 import learned as L
    net = L.Net(seed=2)
    rng = np.random.default_rng(1)
    pred = torch.tensor(rng.standard_normal(1000), dtype=torch.float32, device="cuda")
    targ = torch.tensor(rng.standard_normal(1000), dtype=torch.float32, device="cuda")
    grad = torch.zeros_like(pred)
    loss = net.mse(pred, targ, grad)
    pn, tn = pred.cpu().numpy().astype(np.float64), targ.cpu().numpy().astype(np.float64)
    assert np.isclose(loss, ((pn - tn) ** 2).mean(), rtol=1e-6)
    assert np.allclose(grad.cpu().numpy(), 2 * (pn - tn) / 1000, rtol=1e-5)
    p0 = net.p.clone()
    net.g.copy_(torch.ones_like(net.g))
    net.adam(1e-3)
    # first Adam step moves every parameter by lr (bias-corrected moments of a constant gradient)
    assert np.allclose((p0 - net.p).cpu().numpy(), 1e-3, rtol=1e-3)


def test_trained_guess_gains_iterations():
    """The committed trained network: on a held-out elastic image the guess cuts PCG iterations
    and leaves the tensor unchanged."""
    from chfem_b200 import learned as L
    from chfem_b200 import synthetic
    if not os.path.exists(L.DEFAULT_WEIGHTS):
        pytest.skip("no trained weights committed")
    net = L.Net.load()
    img = synthetic.grf((48, 48, 48), corr=6.0, fraction=0.4, seed=987654)
    props = {0: (1.0, 0.30), 255: (12.0, 0.20)}
    # tolerance 1e-8: two solves stopped at tol agree to O(tol) whatever their starting points
    C0, its0, _, _ = L.solve_elastic(img, props, tol=1e-8, precision="fp64", want_x=False)
    x0 = L.initial_guesses(net, img, props)
    C1, its1, _, _ = L.solve_elastic(img, props, tol=1e-8, precision="fp64", x0=x0, want_x=False)
    assert H.rel_to_max(C1, C0) < 1e-6
    assert sum(its1) < 0.9 * sum(its0), (its1, its0)


@pytest.mark.parametrize("multirhs", [True, False])
def test_compute_property_with_learned_guess(multirhs):
    """compute_property(initial_guess='learned') returns the zero-guess tensor (both solve
    paths take the device-resident guesses)."""
    from chfem_b200 import compute_property
    from chfem_b200 import learned as L
    from chfem_b200 import synthetic
    if not os.path.exists(L.DEFAULT_WEIGHTS):
        pytest.skip("no trained weights committed")
    img = synthetic.grf((40, 48, 32), corr=6.0, fraction=0.4, seed=4242)
    props = {0: (1.0, 0.30), 255: (20.0, 0.20)}
    kw = dict(mat_props=props, solver_tolerance=1e-8, solver_maxiter=20000, multirhs=multirhs)
    C0 = np.array(compute_property("elasticity", img, **kw))
    C1 = np.array(compute_property("elasticity", img, initial_guess="learned", **kw))
    assert H.rel_to_max(C1, C0) < 1e-6
    with pytest.raises(ValueError):
        compute_property("elasticity", img[:, :, :30], initial_guess="learned", **kw)
