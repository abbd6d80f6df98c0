"""The fused SART step (sart_fused_kernel: back projection of view p and forward projection
of view p + 1 in one pass over each volume row) against the unfused kernels
(bp_sart_column_kernel + the xz forward projector): the volumes and residual sums must
be bit-identical, since the fused kernel performs the same operations in the same
order; the fused path must be the one that ran (M + 1 launches per iteration instead of
2 M); and one case is held to the oracle within the column kernel's tolerance."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _context(fused):
    from ettention_b200.operators import Context
    os.environ["ETCU_FUSED"] = "1" if fused else "0"
    try:
        return Context(0)
    finally:
        del os.environ["ETCU_FUSED"]


def _run(fused, res, geoms, projs, params, iters):
    from ettention_b200.operators import BlockIterativeReconstructionOperator, GPUMappedVolume
    ctx = _context(fused)
    try:
        vol = GPUMappedVolume(ctx, res)
        rec = BlockIterativeReconstructionOperator(vol, geoms, projs, params)
        launches = rec.launches_per_iteration
        rec.runNiterations(iters)
        v = rec.getReconstructedVolume()
        last = rec.last_residual_sq()
        rec.close()
        vol.close()
    finally:
        ctx.close()
    return v, last, launches


def _problem(res, det, angles, seed):
    from oracle import oracle as O
    from ettention_b200.operators import mrc_base_geometry
    from tests.helpers import ellipsoid_phantom, oracle_geometry
    X, Y, Z = res
    truth = ellipsoid_phantom(res, 6, seed=seed)
    vg = O.VolumeGeometry.centered(res)
    base = mrc_base_geometry(*det)
    geoms = [base.rotated(float(a)) for a in angles]
    projs = np.stack([O.forward_project(truth, vg, oracle_geometry(g), 1, 32)[0] for g in geoms]).astype(np.float32)
    return geoms, projs


CASES = [
    # volume, detector, angles, order, long-object compensation
    ((128, 64, 48), (128, 64), list(np.linspace(-70, 70, 15)) + [90.0, 0.0], "identity", True),
    ((256, 32, 40), (200, 32), list(np.linspace(-60, 60, 9)), "random", False),
    ((96, 16, 130), (96, 16), [-89.0, -45.0, -1.0, 0.0, 33.3, 60.0, 91.0, 180.0], "maxangle", True),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_fused_step_is_bit_identical_to_unfused(case):
    from ettention_b200.operators import AlgebraicParameterSet, ORDERS
    res, det, angles, order, loc = CASES[case]
    geoms, projs = _problem(res, det, angles, seed=100 + case)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=ORDERS[order],
                              use_long_object_compensation=loc)
    vf, lf, nf = _run(True, res, geoms, projs, p, 2)
    vu, lu, nu = _run(False, res, geoms, projs, p, 2)
    M = len(angles)
    assert nf == M + 1 and nu == 2 * M, (nf, nu)
    assert np.abs(vu).max() > 0
    assert np.array_equal(vf, vu)
    assert lf == pytest.approx(lu, rel=1e-12)  # FP64 sums of the same residuals, atomics in another order


def test_fused_step_against_oracle():
    from oracle import oracle as O
    from ettention_b200 import _abi
    from ettention_b200.operators import AlgebraicParameterSet
    from tests.helpers import oracle_geometry
    res, det = (64, 32, 24), (64, 32)
    angles = list(np.linspace(-60, 60, 11))
    geoms, projs = _problem(res, det, angles, seed=7)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.5, order=_abi.ORDER_IDENTITY)
    v, _, n = _run(True, res, geoms, projs, p, 2)
    assert n == len(angles) + 1
    vg = O.VolumeGeometry.centered(res)
    setup = O.ReconstructionSetup(vg, [oracle_geometry(g) for g in geoms], projs, 0.5, 1, 1, 1)
    vo = np.zeros((res[2], res[1], res[0]), np.float32)
    O.block_iterative(setup, vo, 2, 32)
    assert O.rel_l2(v, vo) <= 1e-4


def test_ineligible_reconstructions_fall_back():
    """Detector taller than the volume (many detector rows clamp onto one volume row),
    SIRT, and a masked volume keep the unfused launches."""
    from ettention_b200.operators import AlgebraicParameterSet, ORDERS
    res = (64, 32, 16)
    geoms, projs = _problem(res, (64, 80), [-30.0, 0.0, 30.0], seed=3)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=1, lam=0.3, order=ORDERS["identity"])
    vf, lf, nf = _run(True, res, geoms, projs, p, 1)
    vu, lu, nu = _run(False, res, geoms, projs, p, 1)
    assert nf == nu == 6
    assert np.array_equal(vf, vu)
    geoms, projs = _problem(res, (64, 32), [-30.0, 0.0, 30.0], seed=4)
    q = AlgebraicParameterSet(algorithm="sirt", block_size=3, iterations=1, lam=0.3, order=ORDERS["identity"])
    _, _, n = _run(True, res, geoms, projs, q, 1)
    assert n == 2
