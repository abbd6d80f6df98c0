"""Convergence of plain SART (the reference's update, BlockIterativeReconstructionOperator.cpp:
92-142, with its ray-driven projector and voxel-driven back projector) in the data residual
||Ax - b||^2, on the FP64 CPU oracle: a 64 x 64 x 32 ellipsoid phantom, 31 parallel views
-60..60 deg, Poisson noise at 100 counts per pixel.

* relaxation 0.3: the residual falls for 3 iterations and then rises without bound, so
  after 30 iterations it is above the residual of the first iteration -- "the time to
  reach plain SART's 30-iteration residual" would be one iteration;
* relaxation 0.05: the residual falls at every one of the first 10 iterations and stays
  within 3 % of its minimum through 30 iterations.

This is why the learned warm start's workload uses a small relaxation (0.03, see
ettention_b200/warmstart.py), where plain SART's residual still falls at iteration 30."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def problem():
    from oracle import oracle as O
    from tests.helpers import ellipsoid_phantom
    res = (64, 64, 32)
    ph = ellipsoid_phantom(res, 12, axes=(2.0, 16.0), density=(0.002, 0.04), seed=77)
    vg = O.VolumeGeometry.centered(res)
    geoms = [O.rotate_geometry(O.mrc_base_geometry(64, 64), float(a)) for a in np.linspace(-60, 60, 31)]
    p = np.stack([O.forward_project(ph, vg, g, 1, 64)[0] for g in geoms]).astype(np.float64)
    rng = np.random.Generator(np.random.PCG64(77))
    b = (-np.log(np.maximum(rng.poisson(100 * np.exp(-p)), 1) / 100)).astype(np.float32)
    return vg, geoms, b


def residuals(problem, lam, iters=30):
    from oracle import oracle as O
    vg, geoms, b = problem
    setup = O.ReconstructionSetup(vg, geoms, b, lam, 1)
    v = np.zeros((32, 64, 64), np.float32)
    out = []
    for _ in range(iters):
        O.block_iterative(setup, v, 1, 64)
        out.append(sum(float(((b[i] - O.forward_project(v, vg, g, 1, 64)[0]).astype(np.float64) ** 2).sum())
                       for i, g in enumerate(geoms)))
    return np.array(out)


def test_relaxation_03_residual_rises(problem):
    r = residuals(problem, 0.3)
    k = int(np.argmin(r))
    assert 1 <= k <= 5, r
    assert r[-1] > 10.0 * r.min()
    assert r[-1] > r[0]  # plain SART "reaches" its 30-iteration residual at iteration 1


def test_relaxation_005_residual_falls(problem):
    r = residuals(problem, 0.05)
    assert np.all(np.diff(r[:10]) < 0), r
    assert r[-1] <= 1.03 * r.min()
