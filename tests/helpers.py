"""Shared fixtures for the tests: golden archives, phantoms, geometry bridges."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# The reference checkout (the directory holding `ettention/`), named by the environment
# variable ETTENTION_REFERENCE; tests that read its files directly skip when it is unset.
REFERENCE = os.environ.get("ETTENTION_REFERENCE", "")


def reference_path(*parts: str) -> str:
    """Path inside the reference checkout, or "" when ETTENTION_REFERENCE is unset."""
    return os.path.join(REFERENCE, *parts) if REFERENCE else ""


def golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def xzy_to_zyx(vol_xzy: np.ndarray) -> np.ndarray:
    """MRC volumes written with ORDER_XZY (framework/test/ProjectionTestBase.h:27) hold
    array[y][z][x]; the projectors use array[z][y][x]."""
    return np.ascontiguousarray(np.transpose(vol_xzy, (1, 0, 2)))


def blob_phantom(background: float = 1.0) -> np.ndarray:
    """ProjectionTestBase::allocateVolume (framework/test/ProjectionTestBase.cpp:70-103) on a
    64^3 volume filled with `background` (1.0 in ForwardProjectionTest.cpp:46-49)."""
    v = np.full((64, 64, 64), background, np.float32)

    def blob(p, r, val):
        p = np.asarray(p, np.float32)
        lo = [int(c) - int(r) for c in p]
        hi = [int(c) + int(r) for c in p]
        for z in range(lo[2], hi[2] + 1):
            for y in range(lo[1], hi[1] + 1):
                for x in range(lo[0], hi[0] + 1):
                    d = np.array([x, y, z], np.float32) - p
                    if float(np.sqrt(np.float32((d * d).sum()))) < r:
                        v[z, y, x] = val

    for x in (16.0, 32.0, 48.0):
        for y in (16.0, 32.0, 48.0):
            for z in (16.0, 32.0, 48.0):
                blob((x, y, z), 1, 16.0)
    for c in (16.0, 32.0, 48.0):
        blob((c, c, c), 3, 16.0)
    return v


def ellipsoid_phantom(res_xyz, k: int, axes=(4.0, 32.0), density=(0.1, 1.0), seed: int = 0) -> np.ndarray:
    """Sum of k ellipsoids: centres uniform in the volume, semi-axes uniform in `axes`
    voxels, uniform random rotation, density uniform in `density`, additive."""
    rng = np.random.Generator(np.random.PCG64(seed))
    X, Y, Z = res_xyz
    vol = np.zeros((Z, Y, X), np.float32)
    zz, yy, xx = np.meshgrid(np.arange(Z) + 0.5, np.arange(Y) + 0.5, np.arange(X) + 0.5, indexing="ij")
    for _ in range(k):
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
        p = np.stack([xx[z0:z1, y0:y1, x0:x1] - c[0], yy[z0:z1, y0:y1, x0:x1] - c[1],
                      zz[z0:z1, y0:y1, x0:x1] - c[2]], -1) @ R
        inside = ((p / a) ** 2).sum(-1) <= 1.0
        vol[z0:z1, y0:y1, x0:x1] += np.float32(d) * inside
    return vol


def oracle_geometry(g):
    """Product ScannerGeometry -> oracle ScannerGeometry (same float values)."""
    from oracle import oracle as O
    return O.ScannerGeometry(np.asarray(g.source, np.float64), np.asarray(g.detector, np.float64),
                             np.asarray(g.hpitch, np.float64), np.asarray(g.vpitch, np.float64), g.width, g.height,
                             bool(g.perspective))


def product_geometry(g):
    from ettention_b200.operators import ScannerGeometry
    return ScannerGeometry([float(x) for x in g.source], [float(x) for x in g.detector], [float(x) for x in g.hpitch],
                           [float(x) for x in g.vpitch], g.width, g.height, bool(g.perspective))


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))
