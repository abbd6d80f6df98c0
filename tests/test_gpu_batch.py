"""Batched reconstruction of independent tilt series of uneven sizes (etcu_batch_*).

Every SART step runs one forward-projection launch and one back-projection launch
over all series; series that have no view at a step sit it out.  Per series the
volume must equal the single-series reconstruction with the same kernels (a
context created with ETCU_BP_COLUMN=0, whose single-view back projector is the
row kernel the batch uses) bit for bit, and the oracle within 1e-3 after the
iterations.  Configurations the batch does not cover are refused with
ETCU_ERR_UNSUPPORTED.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RECON_TOL = 1e-3

SERIES = [  # (X, Y, Z), views
    ((48, 40, 24), 13),
    ((64, 48, 32), 17),
    ((40, 40, 40), 9),
    ((96, 32, 16), 21),
]


@pytest.fixture(scope="module")
def ctx():
    import torch
    from ettention_b200.operators import Context
    assert torch.cuda.is_available()
    old = os.environ.get("ETCU_BP_COLUMN")
    os.environ["ETCU_BP_COLUMN"] = "0"
    try:
        c = Context(0)
    finally:
        if old is None:
            del os.environ["ETCU_BP_COLUMN"]
        else:
            os.environ["ETCU_BP_COLUMN"] = old
    yield c
    c.close()


def make_series(seed):
    from oracle import oracle as O
    from ettention_b200.operators import mrc_base_geometry
    from tests.helpers import ellipsoid_phantom, oracle_geometry
    out = []
    for i, ((X, Y, Z), nv) in enumerate(SERIES):
        truth = ellipsoid_phantom((X, Y, Z), 6, seed=seed + i)
        geoms = [mrc_base_geometry(X, Y).rotated(float(a)) for a in np.linspace(-60, 60, nv)]
        vg = O.VolumeGeometry.centered((X, Y, Z))
        projs = np.stack([O.forward_project(truth, vg, oracle_geometry(g), 1, 32)[0] for g in geoms])
        out.append(((X, Y, Z), geoms, projs))
    return out


def test_batch_equals_single_series_and_matches_oracle(ctx):
    from oracle import oracle as O
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BatchReconstructionOperator,
                                          BlockIterativeReconstructionOperator, GPUMappedVolume)
    from tests.helpers import oracle_geometry
    series = make_series(300)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=_abi.ORDER_IDENTITY)
    vols = [GPUMappedVolume(ctx, shape) for shape, _, _ in series]
    batch = BatchReconstructionOperator([(v, g, pr) for v, (_, g, pr) in zip(vols, series)], p)
    assert batch.launches_per_iteration == 2 * max(len(g) for _, g, _ in series)
    batch.runNiterations(2)
    got = batch.getReconstructedVolumes()
    res = batch.last_residual_sq()
    batch.close()
    for v in vols:
        v.close()
    for i, (shape, geoms, projs) in enumerate(series):
        vol = GPUMappedVolume(ctx, shape)
        rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
        rec.runNiterations(2)
        single = rec.getReconstructedVolume()
        r1 = rec.last_residual_sq()
        rec.close()
        vol.close()
        assert np.array_equal(got[i], single), i
        assert abs(res[i] - r1) <= 1e-12 * r1
        X, Y, Z = shape
        vg = O.VolumeGeometry.centered(shape)
        setup = O.ReconstructionSetup(vg, [oracle_geometry(g) for g in geoms], projs, 0.3, 1, 1, 1)
        vo = np.zeros((Z, Y, X), np.float32)
        O.block_iterative(setup, vo, 2, 32)
        assert O.rel_l2(got[i], vo) <= RECON_TOL


@pytest.mark.parametrize("case", ["block_size", "xaxis_tilt", "half_volume", "subvolumes"])
def test_batch_refuses_what_it_does_not_cover(ctx, case):
    from ettention_b200 import _abi
    from ettention_b200._abi import EttentionError
    from ettention_b200.operators import AlgebraicParameterSet, BatchReconstructionOperator, GPUMappedVolume
    from ettention_b200.operators import mrc_base_geometry
    X, Y, Z = 32, 24, 16
    geoms = [mrc_base_geometry(X, Y).rotated(float(a)) for a in (-30, 0, 30)]
    projs = np.zeros((3, Y, X), np.float32)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=1, lam=0.3, order=_abi.ORDER_IDENTITY)
    kw = {}
    if case == "block_size":
        p.block_size = 2
    elif case == "xaxis_tilt":
        geoms = [mrc_base_geometry(X, Y).rotated(float(a), 20.0) for a in (-30, 0, 30)]
    elif case == "half_volume":
        kw = {"voxel_type": _abi.VOXEL_HALF16}
    else:
        kw = {"subvolume_count": 2}
    vol = GPUMappedVolume(ctx, (X, Y, Z), **kw)
    with pytest.raises(EttentionError) as e:
        BatchReconstructionOperator([(vol, geoms, projs)], p)
    assert e.value.status == _abi.ERR_UNSUPPORTED
    vol.close()


@pytest.mark.parametrize("wide", [False, True])
def test_persistent_batch_equals_single_series(wide):
    """With the fused steps available (the default context), the whole batched iteration is
    one launch (sart_fused_batch_kernel: per series and volume row, the first view's forward
    projection, the fused steps and the last view's back projection, taken as units in
    step-major order; blocks of 128 threads while every row is at most 256 voxels and rays
    wide, of 512 with the wide series).  Per series the volume equals the single-series
    reconstruction bit for bit, including a series of one view, with long-object
    compensation and the random order."""
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BatchReconstructionOperator,
                                          BlockIterativeReconstructionOperator, Context, GPUMappedVolume,
                                          mrc_base_geometry)
    from oracle import oracle as O
    from tests.helpers import ellipsoid_phantom, oracle_geometry
    series = make_series(500)
    truth = ellipsoid_phantom((32, 24, 16), 4, seed=77)
    g1 = [mrc_base_geometry(32, 24).rotated(20.0)]
    series.append(((32, 24, 16), g1, np.stack([O.forward_project(truth, O.VolumeGeometry.centered((32, 24, 16)),
                                                                 oracle_geometry(g1[0]), 1, 32)[0]])))
    if wide:
        truth = ellipsoid_phantom((288, 16, 12), 4, seed=78)
        gw = [mrc_base_geometry(288, 16).rotated(float(a)) for a in (-40.0, -10.0, 25.0, 50.0, 5.0)]
        vw = O.VolumeGeometry.centered((288, 16, 12))
        series.append(((288, 16, 12), gw, np.stack([O.forward_project(truth, vw, oracle_geometry(g), 1, 32)[0]
                                                    for g in gw])))
    ctx = Context(0)
    try:
        for order, loc in ((_abi.ORDER_IDENTITY, False), (_abi.ORDER_RANDOM, True)):
            p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=order,
                                      use_long_object_compensation=loc)
            vols = [GPUMappedVolume(ctx, shape) for shape, _, _ in series]
            batch = BatchReconstructionOperator([(v, g, pr) for v, (_, g, pr) in zip(vols, series)], p)
            assert batch.launches_per_iteration == 1
            batch.runNiterations(2)
            got = batch.getReconstructedVolumes()
            res = batch.last_residual_sq()
            batch.close()
            for v in vols:
                v.close()
            for i, (shape, geoms, projs) in enumerate(series):
                vol = GPUMappedVolume(ctx, shape)
                rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
                rec.runNiterations(2)
                want = rec.getReconstructedVolume()
                wres = rec.last_residual_sq()
                rec.close()
                vol.close()
                assert np.abs(want).max() > 0
                assert np.array_equal(got[i], want), (order, loc, i)
                assert res[i] == pytest.approx(wres, rel=1e-12)
    finally:
        ctx.close()


def test_persistent_batch_wait_gives_up_and_context_survives():
    """The persistent batch's waits are bounded: with row 2 of the first series never
    reporting its first step (ETCU_TEST_WITHHOLD_ROW, a flag nothing else sets), the units
    that need it wait out their limit (1 s) and the run returns an error status instead of
    hanging; the same context then reconstructs a series normally."""
    import time
    from ettention_b200 import _abi
    from ettention_b200._abi import EttentionError
    from ettention_b200.operators import (AlgebraicParameterSet, BatchReconstructionOperator,
                                          BlockIterativeReconstructionOperator, Context, GPUMappedVolume)
    series = make_series(700)[:2]
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=1, lam=0.3, order=_abi.ORDER_IDENTITY)
    os.environ["ETCU_TEST_WITHHOLD_ROW"] = "2"
    try:
        ctx = Context(0)
    finally:
        del os.environ["ETCU_TEST_WITHHOLD_ROW"]
    try:
        vols = [GPUMappedVolume(ctx, shape) for shape, _, _ in series]
        batch = BatchReconstructionOperator([(v, g, pr) for v, (_, g, pr) in zip(vols, series)], p)
        assert batch.launches_per_iteration == 1
        t0 = time.time()
        with pytest.raises(EttentionError, match="waited longer than its limit"):
            batch.runNiterations(1)
        assert time.time() - t0 < 30
        batch.close()
        for v in vols:
            v.close()
        q = AlgebraicParameterSet(algorithm="sirt", block_size=_abi.BLOCK_ALL, iterations=1, lam=0.3,
                                  order=_abi.ORDER_IDENTITY)
        shape, geoms, projs = series[0]
        vol = GPUMappedVolume(ctx, shape)
        rec = BlockIterativeReconstructionOperator(vol, geoms, projs, q)
        rec.run()
        after = rec.getReconstructedVolume()
        rec.close()
        vol.close()
    finally:
        ctx.close()
    ctx2 = Context(0)
    try:
        vol = GPUMappedVolume(ctx2, shape)
        rec = BlockIterativeReconstructionOperator(vol, geoms, projs, q)
        rec.run()
        fresh = rec.getReconstructedVolume()
        rec.close()
        vol.close()
    finally:
        ctx2.close()
    assert np.abs(fresh).max() > 0 and np.array_equal(after, fresh)


@pytest.mark.parametrize("vt", [2, 3])
def test_persistent_batch_with_16bit_shadow(vt):
    """Series held as FP32 masters with FP16 (2) / BF16 (3) shadows run the persistent
    batched iteration (one launch) and equal the single-series persistent reconstruction
    bit for bit; after the run the shadows are refreshed from the masters, so a further
    single-series iteration on a batched volume equals three single-series iterations."""
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BatchReconstructionOperator,
                                          BlockIterativeReconstructionOperator, Context, GPUMappedVolume)
    series = make_series(600)
    ctx = Context(0)
    try:
        p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=_abi.ORDER_IDENTITY)
        vols = [GPUMappedVolume(ctx, shape, voxel_type=vt) for shape, _, _ in series]
        batch = BatchReconstructionOperator([(v, g, pr) for v, (_, g, pr) in zip(vols, series)], p)
        assert batch.launches_per_iteration == 1
        batch.runNiterations(2)
        got = batch.getReconstructedVolumes()
        batch.close()
        for i, (shape, geoms, projs) in enumerate(series):
            vol = GPUMappedVolume(ctx, shape, voxel_type=vt)
            rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
            rec.runNiterations(2)
            assert np.abs(got[i]).max() > 0 and np.array_equal(got[i], rec.getReconstructedVolume()), i
            rec.runNiterations(1)
            want3 = rec.getReconstructedVolume()
            rec.close()
            vol.close()
            cont = BlockIterativeReconstructionOperator(vols[i], geoms, projs, p)
            cont.runNiterations(1)
            assert np.array_equal(cont.getReconstructedVolume(), want3), i
            cont.close()
        for v in vols:
            v.close()
    finally:
        ctx.close()


@pytest.mark.parametrize("kind", [1, 2])
def test_persistent_batch_with_16bit_projections(kind):
    """Tilt series stored in FP16 (1) / BF16 (2) on the persistent batched path (FP16-shadow
    volumes): every series equals its single-series reconstruction with the same storage,
    bit for bit."""
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BatchReconstructionOperator,
                                          BlockIterativeReconstructionOperator, Context, GPUMappedVolume)
    series = make_series(700)
    ctx = Context(0)
    try:
        p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=_abi.ORDER_IDENTITY,
                                  projection_storage=kind)
        vols = [GPUMappedVolume(ctx, shape, voxel_type=2) for shape, _, _ in series]
        batch = BatchReconstructionOperator([(v, g, pr) for v, (_, g, pr) in zip(vols, series)], p)
        assert batch.launches_per_iteration == 1
        batch.runNiterations(2)
        got = batch.getReconstructedVolumes()
        batch.close()
        for v in vols:
            v.close()
        for i, (shape, geoms, projs) in enumerate(series):
            vol = GPUMappedVolume(ctx, shape, voxel_type=2)
            rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
            rec.runNiterations(2)
            assert np.abs(got[i]).max() > 0 and np.array_equal(got[i], rec.getReconstructedVolume()), i
            rec.close()
            vol.close()
    finally:
        ctx.close()
