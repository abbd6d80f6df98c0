"""The fused SART step (back projection of view p and forward projection of view p + 1 in
one pass over each volume row), launched per step (sart_fused_kernel) and as one
persistent launch per iteration (sart_fused_persistent_kernel), against the unfused
kernels (bp_sart_column_kernel + the xz forward projector): the volumes and residual sums
must be bit-identical, since the fused kernels perform the same operations in the same
order; the fused paths must be the ones that ran (3 launches per iteration persistent,
M + 1 per step, 2 M unfused); and one case is held to the oracle within the column
kernel's tolerance."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


MODES = {"persistent": ("1", "1"), "step": ("1", "0"), "unfused": ("0", "0")}


def _context(mode):
    """persistent: all fused steps of an iteration in one launch (sart_fused_persistent_kernel);
    step: one launch per fused step (sart_fused_kernel); unfused: the column BP and xz FP."""
    from ettention_b200.operators import Context
    if mode in (True, False):
        mode = "persistent" if mode else "unfused"
    os.environ["ETCU_FUSED"], os.environ["ETCU_PERSIST"] = MODES[mode]
    try:
        return Context(0)
    finally:
        del os.environ["ETCU_FUSED"]
        del os.environ["ETCU_PERSIST"]


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


def _problem(res, det, angles, seed, vpitch=1.0):
    from oracle import oracle as O
    from ettention_b200.operators import ScannerGeometry, mrc_base_geometry
    from tests.helpers import ellipsoid_phantom, oracle_geometry
    X, Y, Z = res
    truth = ellipsoid_phantom(res, 6, seed=seed)
    vg = O.VolumeGeometry.centered(res)
    base = mrc_base_geometry(*det)
    if vpitch != 1.0:  # detector rows vpitch volume rows apart (rows of rays skip volume rows)
        h = 0.5 * det[1] * vpitch
        base = ScannerGeometry([base.source[0], -h, base.source[2]], [base.detector[0], -h, base.detector[2]],
                               list(base.hpitch), [0.0, vpitch, 0.0], det[0], det[1], False)
    geoms = [base.rotated(float(a)) for a in angles]
    projs = np.stack([O.forward_project(truth, vg, oracle_geometry(g), 1, 32)[0] for g in geoms]).astype(np.float32)
    return geoms, projs


CASES = [
    # volume, detector, angles, order, long-object compensation, detector row pitch
    ((128, 64, 48), (128, 64), list(np.linspace(-70, 70, 15)) + [90.0, 0.0], "identity", True, 1.0),
    ((256, 32, 40), (200, 32), list(np.linspace(-60, 60, 9)), "random", False, 1.0),
    ((96, 16, 130), (96, 16), [-89.0, -45.0, -1.0, 0.0, 33.3, 60.0, 91.0, 180.0], "maxangle", True, 1.0),
    ((64, 40, 24), (64, 16), list(np.linspace(-50, 50, 7)), "random", False, 2.5),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_fused_step_is_bit_identical_to_unfused(case):
    """The persistent launch, the per-step launches and the unfused kernels give the same
    volume bit for bit (the steps of a volume row wait for the rows whose detector rows
    they read or overwrite, so every row sees the same data as in step order)."""
    from ettention_b200.operators import AlgebraicParameterSet, ORDERS
    res, det, angles, order, loc, vpitch = CASES[case]
    geoms, projs = _problem(res, det, angles, seed=100 + case, vpitch=vpitch)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=ORDERS[order],
                              use_long_object_compensation=loc)
    vp, lp, np_ = _run("persistent", res, geoms, projs, p, 2)
    vf, lf, nf = _run("step", res, geoms, projs, p, 2)
    vu, lu, nu = _run("unfused", res, geoms, projs, p, 2)
    M = len(angles)
    assert nu == 2 * M
    if vpitch == 1.0:
        assert nf == M + 1 and np_ == 3, (np_, nf, nu)
    else:
        assert (nf, np_) in ((M + 1, 3), (2 * M, 2 * M)), (np_, nf, nu)
    assert np.abs(vu).max() > 0
    assert np.array_equal(vf, vu)
    assert np.array_equal(vp, vu)
    assert lf == pytest.approx(lu, rel=1e-12)  # FP64 sums of the same residuals, atomics in another order
    assert lp == pytest.approx(lu, rel=1e-12)


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
    assert n == 3  # FP of the first view, the persistent fused steps, BP of the last view
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


def test_persistent_wait_gives_up_and_context_survives():
    """The persistent launch's waits are bounded: with one row's first step never reported
    (ETCU_TEST_WITHHOLD_ROW, a flag nothing sets), the units that need it wait out their
    limit (1 s), the run returns an error status instead of hanging, and the same context
    then runs another reconstruction with results equal to a fresh context's."""
    import time
    from ettention_b200 import _abi
    from ettention_b200._abi import EttentionError
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator, Context,
                                          GPUMappedVolume)
    res, det = (64, 32, 24), (64, 32)
    geoms, projs = _problem(res, det, list(np.linspace(-60, 60, 11)), seed=9)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=1, lam=0.5, order=_abi.ORDER_IDENTITY)
    os.environ["ETCU_FUSED"], os.environ["ETCU_PERSIST"], os.environ["ETCU_TEST_WITHHOLD_ROW"] = "1", "1", "3"
    try:
        ctx = Context(0)
    finally:
        for k in ("ETCU_FUSED", "ETCU_PERSIST", "ETCU_TEST_WITHHOLD_ROW"):
            del os.environ[k]
    try:
        vol = GPUMappedVolume(ctx, res)
        rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
        assert rec.launches_per_iteration == 3
        t0 = time.time()
        with pytest.raises(EttentionError, match="waited longer than its limit"):
            rec.runNiterations(1)
        assert time.time() - t0 < 30
        rec.close()
        vol.close()
        q = AlgebraicParameterSet(algorithm="sirt", block_size=_abi.BLOCK_ALL, iterations=2, lam=0.5,
                                  order=_abi.ORDER_IDENTITY)
        vol = GPUMappedVolume(ctx, res)
        rec = BlockIterativeReconstructionOperator(vol, geoms, projs, q)
        rec.run()
        after = rec.getReconstructedVolume()
        rec.close()
        vol.close()
    finally:
        ctx.close()
    fresh, _, _ = _run("unfused", res, geoms, projs, q, 2)
    assert np.abs(fresh).max() > 0 and np.array_equal(after, fresh)


@pytest.mark.parametrize("vt", [2, 3])
def test_fused_steps_with_16bit_shadow(vt):
    """FP32 master with an FP16 (2) / BF16 (3) shadow on the fused paths: the walk reads
    each updated chunk rounded as the shadow holds it, so the persistent and per-step
    launches and the unfused kernels (the column back projector writing master and shadow,
    the forward projector reading the shadow) give the same volume bit for bit; the FP64
    oracle is met at the storage bound."""
    from oracle import oracle as O
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator,
                                          GPUMappedVolume)
    from tests.helpers import oracle_geometry
    res, det = (128, 64, 48), (128, 64)
    angles = list(np.linspace(-70, 70, 15))
    geoms, projs = _problem(res, det, angles, seed=31)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=_abi.ORDER_IDENTITY)

    def run(mode):
        ctx = _context(mode)
        try:
            vol = GPUMappedVolume(ctx, res, voxel_type=vt)
            rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
            n = rec.launches_per_iteration
            rec.runNiterations(2)
            v = rec.getReconstructedVolume()
            rec.close()
            vol.close()
        finally:
            ctx.close()
        return v, n

    vp, np_ = run("persistent")
    vs, ns = run("step")
    vu, nu = run("unfused")
    M = len(angles)
    assert (np_, ns, nu) == (3, M + 1, 2 * M)
    assert np.abs(vp).max() > 0 and np.array_equal(vp, vs) and np.array_equal(vp, vu)
    vg = O.VolumeGeometry.centered(res)
    setup = O.ReconstructionSetup(vg, [oracle_geometry(g) for g in geoms], projs, 0.3, 1, 1, 1)
    v64 = np.zeros((res[2], res[1], res[0]), np.float32)
    O.block_iterative(setup, v64, 2, 64)
    assert O.rel_l2(vp, v64) <= (1e-2 if vt == 2 else 3e-2)
