"""Trains the learned warm start (macroflow3d_b200.WarmStart) on pairs the solver generates.

    python -m macroflow3d_b200.warmstart_train --pairs 2000 --size 128 --out weights.npy

Pairs: lnK fields from the randomization method (variance drawn uniformly from 0.5-4,
correlation length from 4-12 cells, one seed per pair) and their heads, solved by the batched
mixed-precision CCMG-PCG to ||r||/||b|| <= 1e-10 with h = 1 / 0 on the x faces and no flow
elsewhere.  Training: Adam on minibatches with this library's own forward and backward
kernels, the learning rate decayed by a cosine from `lr` to lr / 10.  The parameters are
saved as FP32 (numpy .npy).
"""
from __future__ import annotations

import argparse
import math
import time

import numpy as np


def generate_pairs(M, n, count, seed, batch=64, sigma2=(0.5, 4.0), lam=(4.0, 12.0), log=print):
    """(lnK, h) FP32 CUDA tensors of `count` solver-generated pairs on an n^3 grid."""
    import torch
    rng = np.random.default_rng(seed)
    g = M.Grid3D(n, n, n, 1.0)
    bc = M.BCSpec.darcy_x()
    cfg = M.HeadSolveConfig(mg_levels=8, cg_rtol=1e-10, cg_check_every=1, conv_norm=M.CONV_B,
                            precision=M.PREC_FP32, cg_max_iter=500)
    stream = torch.cuda.current_stream().cuda_stream
    out_lnK, out_h = [], []
    solver = M.BatchSolver([g] * batch, bc, cfg, stream=stream)
    done = 0
    t0 = time.time()
    while done < count:
        b = min(batch, count - done)
        if b != batch:
            solver.close()
            solver = M.BatchSolver([g] * b, bc, cfg, stream=stream)
        lnKs, Ks = [], []
        for r in range(b):
            s2 = float(rng.uniform(*sigma2))
            lm = float(rng.uniform(*lam))
            lk = M.generate_K_field(g, s2, (lm, lm, lm), seed=int(seed * 100003 + done + r), log_only=True)
            lnKs.append(lk)
            Ks.append(torch.exp(lk))
        hs = [torch.empty_like(K) for K in Ks]
        solver.set_K(Ks)
        res = solver.solve(hs)
        if not all(x.converged for x in res):
            raise RuntimeError("a training solve did not converge")
        for lk, h in zip(lnKs, hs):
            out_lnK.append(lk.float().contiguous())
            out_h.append(h.float().contiguous())
        done += b
        del Ks, hs
    solver.close()
    torch.cuda.synchronize()
    log(f"generated {count} pairs at {n}^3 in {time.time() - t0:.1f} s")
    return out_lnK, out_h


def train(M, ws, n, lnKs, hs, epochs, batch, lr, seed=0, time_budget=None, log=print):
    """Adam on minibatches; returns the per-epoch mean training loss."""
    rng = np.random.default_rng(seed)
    g = M.Grid3D(n, n, n, 1.0)
    bc = M.BCSpec.darcy_x()
    steps_per_epoch = max(1, len(lnKs) // batch)
    total = epochs * steps_per_epoch
    t0 = time.time()
    hist = []
    step = 0
    for ep in range(epochs):
        order = rng.permutation(len(lnKs))
        losses = []
        for k in range(steps_per_epoch):
            idx = order[k * batch:(k + 1) * batch]
            a = lr * (0.1 + 0.9 * 0.5 * (1.0 + math.cos(math.pi * step / max(1, total))))
            losses.append(ws.train_step(g, bc, [lnKs[i] for i in idx], [hs[i] for i in idx], a))
            step += 1
            if time_budget is not None and time.time() - t0 > time_budget:
                break
        hist.append(float(np.mean(losses)))
        log(f"epoch {ep}: loss {hist[-1]:.5f} ({step} steps, {time.time() - t0:.1f} s)")
        if time_budget is not None and time.time() - t0 > time_budget:
            log("time budget reached")
            break
    return hist


def main():
    import torch
    import macroflow3d_b200 as M
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--time-budget", type=float, default=None, help="seconds of training, at most")
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    torch.cuda.set_device(0)
    lnKs, hs = generate_pairs(M, args.size, args.pairs, args.seed)
    ws = M.WarmStart(seed=args.seed)
    train(M, ws, args.size, lnKs, hs, args.epochs, args.batch, args.lr, seed=args.seed,
          time_budget=args.time_budget)
    ws.save(args.out)
    print(f"saved {ws.num_params} parameters to {args.out}")


if __name__ == "__main__":
    main()
