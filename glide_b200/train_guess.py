"""Train the learned initial guess on solutions of the plain FP64 solver.

Usage (GPU):
    python -m glide_b200.train_guess --patches 4000 --epochs 4 --out glide_b200/guess_weights.pt

1. Training data: seeded 256x256 patches (dx = 1 km) of the grounded-dome
   family, each one implicit step (dt = 10 a) from u = v = 0 solved by the
   plain FP64 FAS solver (``precision="fp64"``) to 1e-8 relative residual;
   patches are solved in batches (one batched hierarchy, ``batch=nb``).
2. Inputs (H, bed, beta, B) -> targets (cell-centred u, v) / 100 m/a.
3. The U-Net of ``glide_b200.guess`` is trained with Adam on FP32 master
   weights; every convolution runs on the tcgen05 BF16 GEMM.
Prints one JSON line per phase.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from .guess import GuessModel, UNet, cell_velocities, features
from .physics import IcePhysics
from .solver import SolverSettings
from .synthetic import training_patch_case

TOL_SETTINGS = dict(shift=0.0, err_threshold=1e-7)


def solve_batch(seeds, n=256, levels=4, tol=1e-8, max_vcycles=30):
    cases = [training_patch_case(s, n=n, n_levels=levels) for s in seeds]
    nb = len(cases)
    ph = IcePhysics(n, n, cases[0].dx, n_levels=levels, precision="fp64", batch=nb,
                    settings=SolverSettings(**TOL_SETTINGS))
    st = lambda k: np.stack([getattr(c, k) for c in cases])
    ph.set_geometry(st("bed"), st("thickness"))
    ph.set_parameters(B=st("B"), beta=st("beta"), smb=st("smb"))
    ph.forward(10.0, tol=tol, max_vcycles=max_vcycles)
    g = ph.grid
    x = features(torch.as_tensor(st("thickness"), device="cuda"), torch.as_tensor(st("bed"), device="cuda"),
                 torch.as_tensor(st("beta"), device="cuda"), torch.as_tensor(st("B"), device="cuda"))
    y = cell_velocities(g.u, g.v).float()
    return x, y.to(torch.bfloat16), ph.last_info


def generate(n_patches, batch=16, n=256, seed0=0, log=print):
    xs, ys = [], []
    t0 = time.time()
    infos = []
    for b0 in range(0, n_patches, batch):
        seeds = list(range(seed0 + b0, seed0 + min(b0 + batch, n_patches)))
        x, y, info = solve_batch(seeds, n=n)
        xs.append(x)
        ys.append(y)
        infos.append(info)
    torch.cuda.synchronize()
    dt = time.time() - t0
    rel = [i.get("rel_residual") for i in infos]
    log(json.dumps({"phase": "data", "patches": n_patches, "seconds": dt, "max_rel_residual": max(rel),
                    "mean_vcycles": float(np.mean([i["vcycles"] for i in infos])),
                    "mean_finish_sweeps": float(np.mean([i["finish_sweeps"] for i in infos]))}))
    return torch.cat(xs), torch.cat(ys)


def train(x, y, epochs=4, batch=8, lr=2e-3, val_frac=0.05, seed=0, log=print):
    torch.manual_seed(seed)
    net = UNet().cuda()
    nval = max(1, int(len(x) * val_frac))
    xv, yv = x[:nval], y[:nval]
    xt, yt = x[nval:], y[nval:]
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    steps = epochs * (len(xt) // batch)
    sched = torch.optim.lr_scheduler.OneCycleLR(opt, max_lr=lr, total_steps=max(steps, 1))
    t0 = time.time()
    it = 0
    for ep in range(epochs):
        perm = torch.randperm(len(xt), device="cuda")
        run = 0.0
        for k in range(len(xt) // batch):
            idx = perm[k * batch:(k + 1) * batch]
            pred = net(xt[idx])
            loss = torch.mean((pred - yt[idx].float()) ** 2)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            sched.step()
            run += float(loss.detach())
            it += 1
        with torch.no_grad():
            pv = torch.cat([net(xv[k:k + batch]) for k in range(0, len(xv), batch)])
            vloss = float(torch.mean((pv - yv.float()) ** 2))
            base = float(torch.mean(yv.float() ** 2))
        log(json.dumps({"phase": "train", "epoch": ep, "train_mse": run / max(1, len(xt) // batch),
                        "val_mse": vloss, "val_mse_of_zero_guess": base, "seconds": time.time() - t0}))
    return GuessModel(net)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--patches", type=int, default=4000)
    ap.add_argument("--batch-solve", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    x, y = generate(a.patches, batch=a.batch_solve)
    model = train(x, y, epochs=a.epochs)
    if a.out:
        model.save(a.out)
        print(json.dumps({"phase": "saved", "path": a.out}))


if __name__ == "__main__":
    main()
