"""Trains the learned warm start on pairs made by this library's own SART and writes the
weights file the solver and the benchmark load.

    python -m ettention_b200.train_warmstart --series 2000 --epochs 3 \
        --out ettention_b200/data/warmstart_256x256x128.npz

Everything runs on cuda:0: the phantoms, their projections, the SART pairs (3 -> 30
iterations), and the network's forward, backward and Adam steps on the tensor cores.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--series", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--res", default="256,256,128")
    ap.add_argument("--out", default=None)
    ap.add_argument("--eval", type=int, default=4, help="held-out series to report the judge on")
    args = ap.parse_args(argv)
    import torch
    from ettention_b200 import warmstart as W
    from ettention_b200.learned import WarmStartNet, save_weights
    from ettention_b200.operators import Context
    res = tuple(int(v) for v in args.res.split(","))
    ctx = Context(0)
    t0 = time.time()
    out = W.train(ctx, args.series, args.epochs, lr=args.lr, res=res, batch=args.batch,
                  log=lambda m: print(m, flush=True))
    print(json.dumps({"pair_seconds": out["pair_seconds"], "train_seconds": out["train_seconds"],
                      "steps": out["steps"], "scale": out["scale"], "history": out["history"]}), flush=True)
    if args.out:
        save_weights(args.out, out["params"], out["scale"], series=args.series, epochs=args.epochs, lr=args.lr,
                     res=np.array(res), history=np.array(out["history"]), train_seed0=W.TRAIN_SEED0,
                     input_iters=W.INPUT_ITERS, target_iters=W.TARGET_ITERS, lam=W.LAMBDA)
    # the judge on a few held-out series
    net = WarmStartNet(ctx, res, params=out["params"], scale=out["scale"])
    for j in range(args.eval):
        s = W.make_series(ctx, W.HELDOUT_SEED0 + j, res)
        plain = W.PlainSart(ctx, s)
        plain.set_volume(None)
        r = []
        for _ in range(W.TARGET_ITERS):
            plain.iterate(1)
            r.append(plain.residual())
        plain.close()
        solver = W.WarmStartSolver(ctx, net, s)
        kept = solver.start()
        rw = []
        for _ in range(W.TARGET_ITERS - W.INPUT_ITERS):
            rw.append(solver.residual())
            solver.iterate(1)
        solver.close()
        k = next((i for i, x in enumerate(rw) if x <= r[-1]), None)
        print(json.dumps({"seed": s.seed, "plain_r3": r[W.INPUT_ITERS - 1], "plain_r30": r[-1],
                          "judge": solver.judge, "kept": kept, "warm_residuals": rw[:12],
                          "extra_iters_to_target": k}), flush=True)
    net.close()
    ctx.close()
    print(f"total {time.time() - t0:.1f}s", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
