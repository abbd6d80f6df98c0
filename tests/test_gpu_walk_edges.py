"""Forward projection at the edges of the xz walk's applicability.

The xz walk (parallel views tilted about y) decodes the current voxel from its
offset iz * rx * ry + ix, which needs at least two y rows; a sub-volume one voxel
high takes the general 3-D walk.  Both must match the oracle, for rays entering
through every face (tilts from -90 to 90 degrees, detectors wider than the volume)
and for a SART iteration on a single-slice volume.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP_TOL = 1e-4
RECON_TOL = 1e-3


@pytest.fixture(scope="module")
def ctx():
    import torch
    from ettention_b200.operators import Context
    assert torch.cuda.is_available()
    c = Context(0)
    yield c
    c.close()


def forward(ctx, vol_np, g):
    import torch
    from ettention_b200.operators import ForwardProjectionOperator, GPUMappedVolume
    Z, Y, X = vol_np.shape
    vol = GPUMappedVolume(ctx, (X, Y, Z))
    vol.upload(vol_np)
    fp = ForwardProjectionOperator(vol, 1)
    fp.setScannerGeometry(g)
    p = torch.zeros((g.height, g.width), dtype=torch.float32, device="cuda")
    l = torch.zeros_like(p)
    fp.SetOutput(p, l)
    fp.Execute(0)
    ctx.synchronize()
    out = (p.cpu().numpy(), l.cpu().numpy())
    vol.close()
    return out


@pytest.mark.parametrize("Y", [1, 2, 3])
@pytest.mark.parametrize("angle", [-90.0, -60.0, -7.0, 0.0, 33.0, 90.0])
def test_fp_thin_volumes_match_oracle(ctx, Y, angle):
    from oracle import oracle as O
    from ettention_b200.operators import mrc_base_geometry
    from tests.helpers import oracle_geometry
    X, Z = 72, 40
    rng = np.random.Generator(np.random.PCG64(Y * 100 + int(angle + 90)))
    vol = rng.uniform(0, 1, size=(Z, Y, X)).astype(np.float32)
    g = mrc_base_geometry(X + 24, Y).rotated(angle)  # detector wider than the volume
    p, l = forward(ctx, vol, g)
    po, lo = O.forward_project(vol, O.VolumeGeometry.centered((X, Y, Z)), oracle_geometry(g), 1, 32)
    assert O.rel_l2(p, po) <= FP_TOL and O.rel_l2(l, lo) <= FP_TOL


def test_sart_single_slice_volume_matches_oracle(ctx):
    from oracle import oracle as O
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator,
                                          GPUMappedVolume, mrc_base_geometry)
    from tests.helpers import oracle_geometry
    X, Y, Z = 96, 1, 48
    rng = np.random.Generator(np.random.PCG64(8))
    truth = rng.uniform(0, 1, size=(Z, Y, X)).astype(np.float32)
    geoms = [mrc_base_geometry(X, Y).rotated(float(a)) for a in np.linspace(-60, 60, 21)]
    vg = O.VolumeGeometry.centered((X, Y, Z))
    projs = np.stack([O.forward_project(truth, vg, oracle_geometry(g), 1, 32)[0] for g in geoms])
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=_abi.ORDER_IDENTITY)
    vol = GPUMappedVolume(ctx, (X, Y, Z))
    rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p, use_graph=True)
    rec.runNiterations(2)
    v = rec.getReconstructedVolume()
    rec.close()
    vol.close()
    setup = O.ReconstructionSetup(vg, [oracle_geometry(g) for g in geoms], projs, 0.3, 1, 1, 1)
    vo = np.zeros((Z, Y, X), np.float32)
    O.block_iterative(setup, vo, 2, 32)
    assert O.rel_l2(v, vo) <= RECON_TOL
