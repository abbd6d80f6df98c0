"""Warm-started plain SART on the GPU: series generation, training pairs, training, and the
solver with its residual judge.

Workload (the learned warm start's configuration): 256 x 256 x 128 volumes, sums of 40
seeded ellipsoids (semi-axes 8-64 voxels, densities 0.05-1.0 scaled by 0.02 per voxel),
61 parallel views -60..+60 deg step 2 on a 256 x 256 detector, Poisson noise at 100
counts per pixel then -log, SART (block size 1, identity order, zero initial volume) with
relaxation 0.03 -- the largest of 0.3 / 0.1 / 0.05 / 0.03 / 0.02 / 0.01 for which plain
SART's data residual ||Ax - b||^2 falls at every iteration up to at least iteration 50 on
this data.  With 0.3 and 0.1 the residual rises again after a few iterations (so "the time
plain SART takes to reach its 30-iteration residual" would be one iteration); with 0.05
the 30-iteration residual is within 0.2 % of the lowest residual plain SART reaches at
all (its minimum falls near iteration 33), a target no other starting point can be
expected to reach faster.

Training pairs: the volume after INPUT_ITERS plain SART iterations -> the volume after
TARGET_ITERS iterations, both produced by this library's own SART.

Solver (`WarmStartSolver.solve`): INPUT_ITERS plain iterations, the network, then the
judge: the warm start is kept only when its data residual is below that of the
INPUT_ITERS-iteration volume; otherwise SART continues from the plain volume, which is
exactly plain zero-initialised SART.  Then plain SART iterations follow.
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _abi
from .learned import WarmStartNet, init_params
from .operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator, Context,
                        ForwardProjectionOperator, GPUMappedVolume, mrc_base_geometry)
from .phantom import ellipsoid_phantom

RES = (256, 256, 128)
VIEWS = 61
TILT = 60.0
LAMBDA = 0.03
I0 = 100.0
MU = 0.02
ELLIPSOIDS = 40
AXES = (8.0, 64.0)
INPUT_ITERS = 3
TARGET_ITERS = 30
TRAIN_SEED0 = 500000
HELDOUT_SEED0 = 900000


@dataclass
class Series:
    seed: int
    res: tuple
    geoms: list
    b: object          # CUDA float32 (views, y, x)
    phantom: object = None


def make_series(ctx: Context, seed: int, res: Sequence[int] = RES, keep_phantom: bool = False) -> Series:
    """A seeded phantom, its 61 parallel views and noisy projections (CUDA forward
    projection of the phantom, Poisson(I0 exp(-p)), -log(max(counts, 1) / I0))."""
    import torch
    res = tuple(int(r) for r in res)
    X, Y, Z = res
    dev = torch.device("cuda", ctx.device)
    s = X / 256.0
    phantom = ellipsoid_phantom(seed, dev, res, ELLIPSOIDS, (AXES[0] * s, AXES[1] * s), mu_scale=MU)
    geoms = [mrc_base_geometry(X, Y).rotated(float(a)) for a in np.linspace(-TILT, TILT, VIEWS)]
    vol = GPUMappedVolume(ctx, res)
    vol.upload_device(phantom)
    fp = ForwardProjectionOperator(vol, 1)
    projs = torch.zeros((VIEWS, Y, X), dtype=torch.float32, device=dev)
    scratch = torch.zeros((Y, X), dtype=torch.float32, device=dev)
    for i, g in enumerate(geoms):
        fp.setScannerGeometry(g)
        fp.SetOutput(projs[i], scratch)
        fp.Execute(0)
    ctx.synchronize()
    vol.close()
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    counts = torch.poisson(I0 * torch.exp(-projs), generator=gen)
    b = (-torch.log(torch.clamp(counts, min=1.0) / I0)).contiguous()
    torch.cuda.synchronize(dev)
    return Series(seed, res, geoms, b, phantom if keep_phantom else None)


class PlainSart:
    """Plain SART (lambda LAMBDA, identity order, one CUDA graph per iteration) on one
    series, with the volume exchangeable through device memory."""

    def __init__(self, ctx: Context, series: Series, lam: float = LAMBDA):
        import torch
        self.ctx = ctx
        self.vol = GPUMappedVolume(ctx, series.res)
        X, Y, Z = series.res
        self._zeros = torch.zeros((Z, Y, X), dtype=torch.float32, device=torch.device("cuda", ctx.device))
        torch.cuda.synchronize(self._zeros.device)  # filled on torch's stream, read on the library's
        p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=1, lam=lam, order=_abi.ORDER_IDENTITY)
        self.rec = BlockIterativeReconstructionOperator(self.vol, series.geoms, series.b, p, use_graph=True)

    def set_volume(self, t=None) -> None:
        """The volume from device tensor t, or zero (a device-to-device copy of zeros)."""
        self.vol.upload_device(self._zeros if t is None else t)

    def get_volume(self, t) -> None:
        self.vol.download_device(t)

    def iterate(self, n: int) -> None:
        if n > 0:
            self.rec.runNiterations(n)

    def residual(self) -> float:
        """||Ax - b||^2 of the current volume (plain projector, FP64 sum; synchronises)."""
        return self.rec.data_residual_sq()

    def close(self) -> None:
        self.rec.close()
        self.vol.close()


def sart_pair(ctx: Context, series: Series, stops=(INPUT_ITERS, TARGET_ITERS), lam: float = LAMBDA):
    """Volumes (CUDA float32 (z, y, x)) after each number of plain SART iterations in `stops`."""
    import torch
    X, Y, Z = series.res
    out = []
    s = PlainSart(ctx, series, lam)
    done = 0
    for k in stops:
        s.iterate(k - done)
        done = k
        t = torch.empty((Z, Y, X), dtype=torch.float32, device="cuda")
        s.get_volume(t)
        out.append(t)
    ctx.synchronize()
    s.close()
    return out


def train(ctx: Context, n_series: int, epochs: int, lr: float = 1e-3, res: Sequence[int] = RES,
          seed0: int = TRAIN_SEED0, init_seed: int = 0, log=print, batch: int = 1) -> Dict:
    """Generates `n_series` training pairs with this library's SART, then trains the
    network on them with Adam (cosine schedule from lr to lr / 20).  Pairs are kept on the
    device in FP16.  Returns the parameters, the input scale and the loss history."""
    import torch
    res = tuple(int(r) for r in res)
    X, Y, Z = res
    t0 = time.time()
    inputs = torch.empty((n_series, Z, Y, X), dtype=torch.float16, device="cuda")
    targets = torch.empty_like(inputs)
    for i in range(n_series):
        s = make_series(ctx, seed0 + i, res)
        v3, v30 = sart_pair(ctx, s)
        inputs[i].copy_(v3)
        targets[i].copy_(v30)
        del s, v3, v30
        if (i + 1) % 250 == 0:
            log(f"pairs {i + 1}/{n_series} {time.time() - t0:.1f}s")
    gen_s = time.time() - t0
    # input scale: the RMS of the target volumes (the network works in units of it)
    scale = float(torch.sqrt(torch.mean(targets[: min(64, n_series)].float() ** 2)).item())
    net = WarmStartNet(ctx, res, max_batch=batch, params=init_params(init_seed), scale=scale)
    d_in = torch.empty((batch, Z, Y, X), dtype=torch.float32, device="cuda")
    d_t = torch.empty_like(d_in)
    steps = epochs * (n_series // batch)
    history: List[float] = []
    rng = np.random.Generator(np.random.PCG64(init_seed + 17))
    step = 0
    t1 = time.time()
    for ep in range(epochs):
        perm = rng.permutation(n_series)
        run = []
        for j in range(0, n_series - batch + 1, batch):
            idx = torch.as_tensor(perm[j:j + batch], device="cuda")
            d_in.copy_(inputs.index_select(0, idx).float())
            d_t.copy_(targets.index_select(0, idx).float())
            cur = lr * (0.05 + 0.95 * 0.5 * (1.0 + np.cos(np.pi * step / max(1, steps))))
            want = (step % 50) == 0
            l = net.train_step(d_in, d_t, batch, lr=float(cur), want_loss=want)
            if want:
                run.append(l)
            step += 1
        history.append(float(np.mean(run)) if run else float("nan"))
        log(f"epoch {ep + 1}/{epochs} loss {history[-1]:.5f} {time.time() - t1:.1f}s")
    net.check()
    params = net.get_params()
    net.close()
    return {"params": params, "scale": scale, "history": history, "pair_seconds": gen_s,
            "train_seconds": time.time() - t1, "steps": step}


class WarmStartSolver:
    """Plain SART with the learned warm start and its residual judge on one series."""

    def __init__(self, ctx: Context, net: WarmStartNet, series: Series, lam: float = LAMBDA):
        import torch
        self.ctx = ctx
        self.net = net
        self.sart = PlainSart(ctx, series, lam)
        X, Y, Z = series.res
        self.v_in = torch.empty((1, Z, Y, X), dtype=torch.float32, device="cuda")
        self.v_ws = torch.empty_like(self.v_in)
        self.kept: Optional[bool] = None
        self.judge = (None, None)

    def start(self, input_iters: int = INPUT_ITERS) -> bool:
        """INPUT_ITERS plain iterations from zero, the network, the judge.  Returns whether
        the warm start was kept (the reconstruction then continues from it)."""
        self.sart.set_volume(None)
        self.sart.iterate(input_iters)
        r_plain = self.sart.residual()
        self.sart.get_volume(self.v_in[0])
        self.net.infer(self.v_in, self.v_ws, 1)
        self.sart.set_volume(self.v_ws[0])
        r_ws = self.sart.residual()
        self.kept = r_ws < r_plain
        if not self.kept:
            self.sart.set_volume(self.v_in[0])
        self.judge = (r_plain, r_ws)
        return self.kept

    def iterate(self, n: int) -> None:
        self.sart.iterate(n)

    def residual(self) -> float:
        return self.sart.residual()

    def close(self) -> None:
        self.sart.close()
