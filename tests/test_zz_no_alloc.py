"""GPU test of etcu_sart_view_update_noalloc, the allocation-free single-view SART
update for callers that cannot allocate device memory (their memory is reserved up
front by their own pool allocator, or their processing loop may not allocate after
start-up).  It must give the same volume and residual as the allocating
reconstruction entry point (one view, block size 1), on two calls in a row, in each
of its three back-projection branches:

* a parallel view with 4 samples per voxel (the general per-voxel kernel);
* a parallel view tilted about y with one sample per voxel (the single-view row kernel);
* a perspective view (the perspective kernel, sampling factor from the detector size).

Collected last on purpose (file name), so a failing run stops after every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4  # back-projection tolerance of the parity tests (relative L2)


def _geometry(kind, X, Y):
    from ettention_b200.operators import ScannerGeometry, mrc_base_geometry
    if kind == "perspective":
        D = 10.0 * X
        p = 1.0 / D
        base = ScannerGeometry([0.0, 0.0, D], [-0.5 * X * p, -0.5 * Y * p, D - 1.0], [p, 0.0, 0.0], [0.0, p, 0.0],
                               X, Y, True)
        return base.rotated(-17.0)
    return mrc_base_geometry(X, Y).rotated(23.0)


@pytest.mark.parametrize("kind,fp_samples,bp_samples", [("parallel", 2, 4), ("parallel", 1, 1),
                                                        ("perspective", 1, 1)])
def test_noalloc_view_update_matches_allocating_path(kind, fp_samples, bp_samples):
    import torch
    from ettention_b200 import _abi
    from ettention_b200._abi import lib
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator, Context,
                                          GPUMappedVolume)
    from tests.helpers import ellipsoid_phantom

    assert torch.cuda.is_available()
    X, Y, Z = 96, 80, 40
    rng = np.random.Generator(np.random.PCG64(21))
    init = ellipsoid_phantom((X, Y, Z), 8, seed=21) * np.float32(0.5)
    g = _geometry(kind, X, Y)
    b = rng.uniform(0.0, 8.0, (1, Y, X)).astype(np.float32)
    ctx = Context(0)
    try:
        params = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=1, lam=0.4,
                                       order=_abi.ORDER_IDENTITY, fp_samples=fp_samples, bp_samples=bp_samples)
        ref_vol = GPUMappedVolume(ctx, (X, Y, Z))
        ref_vol.upload(init)
        rec = BlockIterativeReconstructionOperator(ref_vol, [g], b, params, use_graph=False)
        na_vol = GPUMappedVolume(ctx, (X, Y, Z))
        na_vol.upload(init)
        d_b = torch.as_tensor(b[0]).cuda()
        torch.cuda.synchronize()
        view = g.to_view()
        stream = ctx.stream_handle
        for call in range(2):
            rec.runNiterations(1)
            ref = rec.getReconstructedVolume()
            ref_r2 = rec.last_residual_sq()
            r2 = ctypes.c_double(-1.0)
            st = lib().etcu_sart_view_update_noalloc(ctypes.byref(ref_vol.desc), na_vol.device_ptr(),
                                                     d_b.data_ptr(), ctypes.byref(view), fp_samples, bp_samples,
                                                     0.4, stream, ctypes.byref(r2))
            assert st == _abi.OK, lib().etcu_last_error(None)
            ctx.synchronize()
            got = na_vol.download()
            d = np.linalg.norm((got - ref).ravel()) / np.linalg.norm((ref - init).ravel())
            assert d <= TOL, f"{kind} call {call}: rel-L2 {d}"
            # the first call projects the same volume (same kernel, sums equal up to the FP64
            # atomics' order); later calls project volumes that agree within TOL (the
            # allocating path's single-view back projector may be another kernel)
            assert abs(r2.value - ref_r2) <= (1e-9 if call == 0 else 1e-6) * ref_r2, (call, r2.value, ref_r2)
        # sizes beyond the static scratch are rejected before any launch: too many pixels,
        # and a narrow detector whose zero-bordered image does not fit (4100 x 260 texels)
        for w, h in ((2048, 1024), (4096, 256)):
            big = _geometry("parallel", w, h).to_view()
            st = lib().etcu_sart_view_update_noalloc(ctypes.byref(ref_vol.desc), na_vol.device_ptr(),
                                                     d_b.data_ptr(), ctypes.byref(big), 1, 1, 0.4, stream, None)
            assert st == _abi.ERR_INVALID_ARGUMENT
            assert b"exceeds" in lib().etcu_last_error(None)
        rec.close()
    finally:
        ctx.close()
