"""Train the learned initial guess (chfem_b200/learned.py) on solutions chfem_b200 computes.

  python -m chfem_b200.train_learned --samples 2000 --epochs 8 --out weights.bin --log log.json

Data: periodic two-phase Gaussian-random-field images (correlation length 6 voxels, 40 %
phase 1) of edge `--size`, phase 0 E = 1, nu = 0.30, phase 1 E log-uniform in [2, 50],
nu = 0.20, seed 5000 + sample.  Each is homogenized with the native block solver (all six load
cases, mixed precision, tolerance --tol); the targets are the periodic fluctuations of the six
solutions.  The network is trained by its own CUDA kernels (forward, backward, Adam) on the
MSE of the fluctuations; the last --holdout samples are never trained on and measure the
validation error and the PCG iterations saved against the zero guess.
"""
import argparse
import json
import math
import time

import numpy as np


def make_sample(i, size, rng):
    from . import synthetic
    img = synthetic.grf((size, size, size), corr=6.0, fraction=0.40, seed=5000 + i)
    ratio = float(math.exp(rng.uniform(math.log(2.0), math.log(50.0))))
    return img, {0: (1.0, 0.30), 255: (ratio, 0.20)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=2000)
    ap.add_argument("--holdout", type=int, default=64)
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--tol", type=float, default=1e-5)
    ap.add_argument("--gen-seconds", type=float, default=1e9, help="stop generating data after this long")
    ap.add_argument("--out", required=True)
    ap.add_argument("--log", default=None)
    args = ap.parse_args(argv)

    import torch
    from . import learned as L
    rng = np.random.default_rng(5000)
    size = args.size
    S = size ** 3
    feats = torch.zeros((args.samples, 2, size, size, size), device="cuda")
    targs = torch.zeros((args.samples, L.OUT_CH, size, size, size), device="cuda")
    meta = []
    t0 = time.time()
    n = 0
    for i in range(args.samples):
        if time.time() - t0 > args.gen_seconds:
            break
        img, props = make_sample(i, size, rng)
        C, its, xs, dev = L.solve_elastic(img, props, tol=args.tol, precision="mixed")
        feats[i] = L.features([img], [props])[0]
        targs[i] = torch.tensor(L.fluctuation(xs, (size, size, size)), device="cuda")
        meta.append({"E1": props[255][0], "iterations": [int(v) for v in its]})
        n += 1
        if n % 100 == 0:
            print(f"generated {n} samples ({time.time() - t0:.0f} s)", flush=True)
    gen_s = time.time() - t0
    hold = min(args.holdout, n // 4)
    ntrain = n - hold
    scale = float(targs[:ntrain].std().item())
    print(f"data: {n} samples ({ntrain} train, {hold} held out) in {gen_s:.0f} s; target std {scale:.3f}", flush=True)

    net = L.Net(seed=1)
    B = args.batch
    steps_per_epoch = ntrain // B
    total = steps_per_epoch * args.epochs
    g = torch.zeros((B, L.OUT_CH, size, size, size), device="cuda")
    history = []
    t1 = time.time()
    step = 0
    for ep in range(args.epochs):
        perm = torch.randperm(ntrain, device="cuda")
        tl = 0.0
        for b in range(steps_per_epoch):
            idx = perm[b * B:(b + 1) * B]
            x = feats[idx].contiguous()
            y = targs[idx].contiguous()
            out = net.forward(x)
            tl += net.mse(out, y, g)
            net.backward(g)
            lr = 0.5 * args.lr * (1 + math.cos(math.pi * step / max(1, total))) + 1e-5
            net.adam(lr)
            step += 1
        # validation: relative L2 error of the fluctuations on the held-out samples
        rel = []
        for j in range(ntrain, n):
            out = net.forward(feats[j:j + 1].contiguous())
            rel.append(float(((out - targs[j:j + 1]).norm() / targs[j:j + 1].norm()).item()))
        history.append({"epoch": ep + 1, "train_mse": tl / max(1, steps_per_epoch), "holdout_rel_error": float(np.mean(rel)),
                        "seconds": time.time() - t1})
        print(json.dumps(history[-1]), flush=True)
    train_s = time.time() - t1
    net.save(args.out)

    # what the guess saves: PCG iterations from the learned vs the zero guess on held-out images
    gains = []
    for j in range(ntrain, min(n, ntrain + 8)):
        img, props = make_sample(j, size, np.random.default_rng(0))
        props = {0: (1.0, 0.30), 255: (meta[j]["E1"], 0.20)}
        C0, its0, _, t0s = L.solve_elastic(img, props, tol=1e-6, precision="fp64", want_x=False)
        x0 = L.initial_guesses(net, img, props)
        C1, its1, _, t1s = L.solve_elastic(img, props, tol=1e-6, precision="fp64", x0=x0, want_x=False)
        gains.append({"sample": j, "iterations_zero": its0, "iterations_learned": its1,
                      "tensor_rel_diff": float(np.abs(C1 - C0).max() / np.abs(C0).max())})
        print(json.dumps(gains[-1]), flush=True)
    log = {"samples": n, "train": ntrain, "holdout": hold, "size": size, "tol": args.tol, "generation_s": gen_s,
           "training_s": train_s, "steps": step, "batch": B, "epochs": args.epochs, "lr": args.lr, "target_std": scale,
           "history": history, "gains": gains,
           "mean_iteration_ratio": float(np.mean([sum(gg["iterations_learned"]) / sum(gg["iterations_zero"]) for gg in gains]))
           if gains else None}
    if args.log:
        with open(args.log, "w") as f:
            json.dump(log, f, indent=1)
    print(json.dumps({k: log[k] for k in ("samples", "generation_s", "training_s", "mean_iteration_ratio")}), flush=True)


if __name__ == "__main__":
    main()
