"""Seeded ellipsoid phantoms on the GPU (synthetic test objects of the benchmark and
training workloads; no dataset is involved)."""
from __future__ import annotations

from typing import Sequence, Tuple

import numpy as np


def ellipsoid_phantom(seed: int, device, res: Sequence[int], count: int, axes: Tuple[float, float],
                      density: Tuple[float, float] = (0.05, 1.0), mu_scale: float = 0.01):
    """Sum of `count` ellipsoids on an (x, y, z) = `res` grid, returned as a float32 torch
    tensor (z, y, x): centres uniform in the volume, semi-axes U(axes) voxels, a uniform
    random rotation (unit quaternion), density U(density) times `mu_scale`, additive.
    numpy PCG64(seed) draws the parameters in that order per ellipsoid."""
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    X, Y, Z = (int(r) for r in res)
    vol = torch.zeros((Z, Y, X), dtype=torch.float32, device=device)
    for _ in range(count):
        c = rng.uniform([0, 0, 0], [X, Y, Z])
        a = rng.uniform(axes[0], axes[1], 3)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        d = rng.uniform(density[0], density[1])
        r = int(np.ceil(a.max())) + 1
        x0, x1 = max(0, int(c[0]) - r), min(X, int(c[0]) + r + 1)
        y0, y1 = max(0, int(c[1]) - r), min(Y, int(c[1]) + r + 1)
        z0, z1 = max(0, int(c[2]) - r), min(Z, int(c[2]) + r + 1)
        if x0 >= x1 or y0 >= y1 or z0 >= z1:
            continue
        zz = torch.arange(z0, z1, device=device, dtype=torch.float32) + 0.5 - float(c[2])
        yy = torch.arange(y0, y1, device=device, dtype=torch.float32) + 0.5 - float(c[1])
        xx = torch.arange(x0, x1, device=device, dtype=torch.float32) + 0.5 - float(c[0])
        Rt = torch.tensor(R, dtype=torch.float32, device=device)
        at = torch.tensor(a, dtype=torch.float32, device=device)
        for zc in range(0, z1 - z0, 64):  # z chunks bound the temporary (chunk, y, x, 3) tensor
            zs = zz[zc:zc + 64]
            p = (xx[None, None, :, None] * Rt[0] + yy[None, :, None, None] * Rt[1] + zs[:, None, None, None] * Rt[2])
            inside = ((p / at) ** 2).sum(-1) <= 1.0
            vol[z0 + zc:z0 + zc + zs.numel(), y0:y1, x0:x1] += float(d * mu_scale) * inside.float()
    return vol
