"""Blob basis functions on the GPU (etcu_forward_project_blobs, etcu_back_project_blobs,
etcu_blob_voxelize, etcu_blob_recon_*) against the oracle and the reference's fixtures:

- forward projection within rel-L2 1e-5 of the oracle (max error 1e-4 of the image's
  maximum), and the 128^3 traversal lengths within ImageComparator's RMS bound of
  intersection_lengths_blobs_reference.tif;
- back projection within rel-L2 1e-4 of the oracle's update (masks included);
- voxelisation bit-exact (the kernel sums in the reference's order);
- the blob forward projection of a blob back projection of projection_reference.tif within
  the reference's RMS bound 0.4 (ForwardProjectionTest.cpp:306-338);
- blob SART / block iterations within rel-L2 1e-4 of the oracle's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP_TOL = 1e-5
BP_TOL = 1e-4


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "the gpu tests need a CUDA device"
    return t


@pytest.fixture(scope="module")
def ctx(torch):
    from ettention_b200.operators import Context
    c = Context(0)
    yield c
    c.close()


def _base(width=64, dist=320.0):
    from ettention_b200.operators import ScannerGeometry
    pitch = 0.1 / width
    return ScannerGeometry([0.0, 0.0, -dist], [-0.05, -0.05, -dist + 1.0], [pitch, 0, 0], [0, pitch, 0], width, width,
                           True)


def _fp_cuda(torch, ctx, vol_np, g, count=256, subvolumes=1):
    from ettention_b200.operators import BlobParameters, GPUMappedVolume, forward_project_blobs
    Z, Y, X = vol_np.shape
    vol = GPUMappedVolume(ctx, (X, Y, Z), subvolume_count=subvolumes)
    vol.upload(vol_np)
    proj = torch.zeros((g.height, g.width), dtype=torch.float32, device="cuda")
    trav = torch.zeros_like(proj)
    forward_project_blobs(vol, g, BlobParameters(), proj, trav, sample_count=count)
    ctx.synchronize()
    vol.close()
    return proj.cpu().numpy(), trav.cpu().numpy()


@pytest.mark.parametrize("angle,subvolumes", [(0.0, 1), (25.0, 3), (70.0, 1), (-115.0, 2)])
def test_fp_vs_oracle(torch, ctx, angle, subvolumes):
    from oracle import oracle as O
    from tests.helpers import oracle_geometry
    g = _base().rotated(angle)
    rng = np.random.default_rng(int(angle) + 200)
    v = rng.uniform(0, 1, size=(40, 44, 48)).astype(np.float32)
    p, L = _fp_cuda(torch, ctx, v, g, 256, subvolumes)
    po, lo = O.forward_project_blobs(v, O.VolumeGeometry.centered((48, 44, 40)), oracle_geometry(g), O.BlobParameters(),
                                     256)
    assert lo.max() > 0
    assert O.rel_l2(p, po) <= FP_TOL and O.rel_l2(L, lo) <= FP_TOL
    assert np.abs(p - po).max() <= 1e-4 * np.abs(po).max()


def test_fp_lengths_golden(torch, ctx):
    """ForwardProjectionTest.cpp PerspectiveBlobs (128-entry table): the traversal lengths
    against the reference's fixture (RMS < 0.1) and the oracle (rel-L2 1e-5)."""
    from oracle import oracle as O
    from tests.helpers import golden, product_geometry
    og = O.perspective_test_geometry()
    ones = np.ones((128, 128, 128), np.float32)
    _, L = _fp_cuda(torch, ctx, ones, product_geometry(og), 128)
    ref = golden("blobs")["intersection_lengths"]
    assert O.rms(L, ref) < 0.1
    _, lo = O.forward_project_blobs(ones, O.VolumeGeometry.centered((128, 128, 128)), og, O.BlobParameters(), 128)
    assert O.rel_l2(L, lo) <= FP_TOL


@pytest.mark.parametrize("angle,block,masked", [(0.0, 1, False), (25.0, 3, False), (-60.0, 1, True)])
def test_bp_vs_oracle(torch, ctx, angle, block, masked):
    from oracle import oracle as O
    from tests.helpers import oracle_geometry
    from ettention_b200.operators import BlobParameters, GPUMappedVolume, back_project_blobs
    g = _base().rotated(angle)
    og = oracle_geometry(g)
    vg = O.VolumeGeometry.centered((48, 44, 40))
    rng = np.random.default_rng(block + 11)
    init = rng.uniform(0, 1, size=(40, 44, 48)).astype(np.float32)
    _, L = O.forward_project_blobs(np.ones_like(init), vg, og, O.BlobParameters(), 256)
    res = rng.normal(size=(64, 64)).astype(np.float32)
    res[rng.uniform(size=res.shape) < 0.1] = 0.0  # zero residuals are skipped
    mask = rng.integers(0, 256, size=init.shape, dtype=np.uint8) if masked else None
    vol = GPUMappedVolume(ctx, (48, 44, 40))
    vol.upload(init)
    if masked:
        vol.set_mask(mask)
    d_res = torch.tensor(res, device="cuda")
    d_len = torch.tensor(L, device="cuda")
    back_project_blobs(vol, g, BlobParameters(), d_res, d_len, 0.7, block)
    got = vol.download()
    vol.close()
    want = init.copy()
    O.back_project_blobs(want, vg, og, res, L, float(np.float32(0.7) / np.float32(block)), O.BlobParameters(),
                         mask=mask)
    assert np.abs(want - init).max() > 0
    assert O.rel_l2(got - init, want - init) <= BP_TOL


def test_forward_matches_back_golden(torch, ctx):
    """ForwardProjectionTest.cpp PerspectiveForwardBlobsMatchesBack: blob back projection
    (lambda 1) of projection_reference.tif with the blob lengths fixture into a zero 128^3
    volume, then the blob forward projection (128-entry table): RMS against the input < 0.4."""
    from oracle import oracle as O
    from tests.helpers import golden, product_geometry
    from ettention_b200.operators import BlobParameters, GPUMappedVolume, back_project_blobs, forward_project_blobs
    g = product_geometry(O.perspective_test_geometry())
    proj = golden("persp")["projection"]
    lengths = golden("blobs")["intersection_lengths"]
    vol = GPUMappedVolume(ctx, (128, 128, 128))
    back_project_blobs(vol, g, BlobParameters(), torch.tensor(proj, device="cuda"),
                       torch.tensor(lengths, device="cuda"), 1.0, 1)
    out = torch.zeros((128, 128), dtype=torch.float32, device="cuda")
    trav = torch.zeros_like(out)
    forward_project_blobs(vol, g, BlobParameters(), out, trav, sample_count=128)
    ctx.synchronize()
    vol.close()
    assert O.rms(out.cpu().numpy(), proj) < 0.4


def test_voxelize_golden_and_oracle(torch, ctx):
    from oracle import oracle as O
    from tests.helpers import golden
    from ettention_b200.operators import BlobParameters, BlobVoxelizerOperator, GPUMappedVolume
    b = np.zeros((16, 16, 16), np.float32)
    b[5, 4, 3] = 1.0
    vol = GPUMappedVolume(ctx, (16, 16, 16))
    vol.upload(b)
    vox = BlobVoxelizerOperator(vol, BlobParameters.createDefault())
    vox.voxelize()
    assert np.array_equal(vox.getVoxelVolume().download(), golden("blobs")["voxelized"])
    vox.getVoxelVolume().close()
    vol.close()
    rng = np.random.default_rng(5)
    r = rng.normal(size=(20, 24, 28)).astype(np.float32)
    vol = GPUMappedVolume(ctx, (28, 24, 20))
    vol.upload(r)
    p = BlobParameters.createWithParameters(1.5, 0, 6.0)
    vox = BlobVoxelizerOperator(vol, p)
    vox.voxelize()
    assert np.array_equal(vox.getVoxelVolume().download(),
                          O.blob_voxelize(r, O.blob_voxelization_kernel(O.BlobParameters(1.5, 0, 6.0))))
    vox.getVoxelVolume().close()
    vol.close()


def _series(n_views=6):
    from oracle import oracle as O
    from tests.helpers import oracle_geometry
    base = _base(32, 160.0)
    geoms = [base.rotated(a) for a in np.linspace(-50, 50, n_views)]
    vg = O.VolumeGeometry.centered((24, 24, 24))
    truth = np.zeros((24, 24, 24), np.float32)
    truth[6:18, 8:16, 9:15] = 1.0
    truth[10:13, 10:13, 4:20] += 0.5
    proj = np.stack([O.forward_project_blobs(truth, vg, oracle_geometry(g), O.BlobParameters(), 256)[0]
                     for g in geoms])
    return geoms, vg, proj


@pytest.mark.parametrize("block", [1, 3])
def test_blob_recon_vs_oracle(torch, ctx, block):
    from oracle import oracle as O
    from tests.helpers import oracle_geometry
    from ettention_b200 import _abi
    from ettention_b200.operators import AlgebraicParameterSet, BlockIterativeReconstructionOperator, GPUMappedVolume
    geoms, vg, proj = _series()
    p = AlgebraicParameterSet(algorithm="sart" if block == 1 else "blockiterative", block_size=block, iterations=2,
                              lam=0.5, order=_abi.ORDER_IDENTITY, basis_functions="blobs")
    vol = GPUMappedVolume(ctx, (24, 24, 24))
    rec = BlockIterativeReconstructionOperator(vol, geoms, proj, p)
    assert rec.view_order() == list(range(len(geoms)))
    rec.run()
    got = rec.getReconstructedVolume()
    rsq = rec.last_residual_sq()
    assert rec.launches_per_iteration == 3 * len(geoms)
    fp_ms, bp_ms, nf, nb = rec.profile_iteration()  # one more iteration, timed per launch
    assert nf == nb == len(geoms) and fp_ms > 0 and bp_ms > 0
    rec.close()
    vol.close()
    want = np.zeros((24, 24, 24), np.float32)
    wsq = O.blob_block_iterations(want, vg, [oracle_geometry(g) for g in geoms], proj, list(range(len(geoms))),
                                  block, 0.5, O.BlobParameters(), iterations=2)
    assert np.abs(want).max() > 0
    assert O.rel_l2(got, want) <= BP_TOL
    assert rsq == pytest.approx(wsq, rel=1e-4)


def test_blob_recon_voxelized_result(torch, ctx):
    """output.options.enableVoxelization: the reconstruction's result is the voxelised
    coefficient volume (BlockIterativeReconstructionOperator.cpp:66-87)."""
    from oracle import oracle as O
    from ettention_b200 import _abi
    from ettention_b200.operators import AlgebraicParameterSet, BlockIterativeReconstructionOperator, GPUMappedVolume
    geoms, _, proj = _series(4)
    p = AlgebraicParameterSet(algorithm="sart", iterations=1, lam=0.5, order=_abi.ORDER_IDENTITY,
                              basis_functions="blobs", enable_voxelization=True)
    vol = GPUMappedVolume(ctx, (24, 24, 24))
    rec = BlockIterativeReconstructionOperator(vol, geoms, proj, p)
    rec.run()
    coefficients = vol.download()
    voxels = rec.getReconstructedVolume()
    rec.close()
    vol.close()
    assert np.abs(coefficients).max() > 0
    assert np.array_equal(voxels, O.blob_voxelize(coefficients, O.blob_voxelization_kernel(O.BlobParameters())))


def test_blob_recon_errors(torch, ctx):
    from ettention_b200 import _abi
    from ettention_b200._abi import EttentionError
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator,
                                          GPUMappedVolume, mrc_base_geometry)
    geoms, _, proj = _series(3)
    p = AlgebraicParameterSet(algorithm="sart", lam=0.5, basis_functions="blobs")
    vol = GPUMappedVolume(ctx, (24, 24, 24))
    par = [mrc_base_geometry(32, 32).rotated(a) for a in (-10.0, 0.0, 10.0)]
    with pytest.raises(EttentionError, match="No fitting forward projection kernel found!"):
        BlockIterativeReconstructionOperator(vol, par, proj, p)
    p.use_long_object_compensation = True
    with pytest.raises(EttentionError, match="only supported for parallel"):
        BlockIterativeReconstructionOperator(vol, geoms, proj, p)
    vol.close()
    p.use_long_object_compensation = False
    half = GPUMappedVolume(ctx, (24, 24, 24), voxel_type=_abi.VOXEL_HALF16)
    with pytest.raises(EttentionError) as e:
        BlockIterativeReconstructionOperator(half, geoms, proj, p)
    assert e.value.status == _abi.ERR_UNSUPPORTED
    half.close()
