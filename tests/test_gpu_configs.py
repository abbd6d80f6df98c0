"""End-to-end parity of the benchmark configurations at small sizes (CUDA path through the
C ABI against the CPU oracle).

* Perspective block-iterative (the 2048^2 x 512 perspective workload, shrunk): perspective
  views with the source at 10 x the volume width, block size 8 with a ragged last block,
  seeded random order, two z sub-volumes whose 22-voxel slabs end in a partial z chunk of
  the perspective back projector, Poisson noise at 200 counts, lambda 0.2.
  FP32 volume against the FP32 oracle (<= 1e-3 after 2 iterations); BF16 shadow with FP32
  master against the FP64 oracle at the BF16 storage bound.
* Parallel SART / SIRT (the 1024^2 x 256 workload, shrunk): 61 views -60..60, Poisson noise
  at 100 counts; SIRT FP32 against the FP32 oracle; SART and SIRT with an FP16 shadow and
  FP32 master against the FP64 oracle at the FP16 storage bound.

Reference loop: BlockIterativeReconstructionOperator.cpp:92-142; perspective back
projection: ocl_src/PerspectiveBeamsBackProjection.cl:28-70.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RECON_TOL = 1e-3      # FP32 path vs FP32 oracle after N iterations (relative L2)
BF16_TOL = 3e-2       # BF16 shadow + FP32 master vs FP64 oracle (8-bit mantissa storage)
F16_TOL = 1e-2        # FP16 shadow + FP32 master vs FP64 oracle (11-bit mantissa storage)


@pytest.fixture(scope="module")
def ctx():
    import torch
    assert torch.cuda.is_available(), "the gpu tests need a CUDA device"
    from ettention_b200.operators import Context
    c = Context(0)
    yield c
    c.close()


def perspective_view(res, tilt):
    """Source 10 x volume width above the centre, detector plane one unit from the source,
    pitch 1 / D so the detector spans the volume at its centre, rotated by -tilt about y."""
    from ettention_b200.operators import ScannerGeometry
    X, Y = res[0], res[1]
    D = 10.0 * X
    p = 1.0 / D
    base = ScannerGeometry([0.0, 0.0, D], [-0.5 * X * p, -0.5 * Y * p, D - 1.0], [p, 0.0, 0.0], [0.0, p, 0.0],
                           X, Y, True)
    return base.rotated(tilt)


def noisy_projections(phantom, geoms, res, i0, seed):
    """FP64 oracle line integrals, Poisson counts at i0 per pixel, then -log."""
    from oracle import oracle as O
    from tests.helpers import oracle_geometry
    vg = O.VolumeGeometry.centered(res)
    p = np.stack([O.forward_project(phantom, vg, oracle_geometry(g), 1, 64)[0] for g in geoms]).astype(np.float64)
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = rng.poisson(i0 * np.exp(-p))
    return (-np.log(np.maximum(counts, 1) / i0)).astype(np.float32)


def cuda_recon(ctx, geoms, projs, res, params, iters, voxel_type=0, subvolumes=1):
    from ettention_b200.operators import BlockIterativeReconstructionOperator, GPUMappedVolume
    vol = GPUMappedVolume(ctx, res, voxel_type=voxel_type, subvolume_count=subvolumes)
    rec = BlockIterativeReconstructionOperator(vol, geoms, projs, params)
    rec.runNiterations(iters)
    out = rec.getReconstructedVolume()
    order = rec.view_order()
    rec.close()
    vol.close()
    return out, order


def oracle_recon(geoms, projs, res, lam, block, iters, order, prec, subvolumes=1):
    from oracle import oracle as O
    from tests.helpers import oracle_geometry
    vg = O.VolumeGeometry.centered(res, subvolumes=subvolumes)
    setup = O.ReconstructionSetup(vg, [oracle_geometry(geoms[i]) for i in order], projs[order], lam, block, 1, 1)
    X, Y, Z = res
    v = np.zeros((Z, Y, X), np.float32)
    O.block_iterative(setup, v, iters, prec)
    return v


PERSP_RES = (96, 96, 44)


@pytest.fixture(scope="module")
def perspective_problem():
    from tests.helpers import ellipsoid_phantom
    res = PERSP_RES
    phantom = ellipsoid_phantom(res, 30, axes=(3.0, 24.0), density=(0.002, 0.02), seed=3001)
    geoms = [perspective_view(res, float(a)) for a in np.linspace(-60.0, 60.0, 31)]
    return geoms, noisy_projections(phantom, geoms, res, 200.0, 3001)


@pytest.mark.parametrize("voxel_type", [0, 3])
def test_perspective_block8_random_order_subvolumes(ctx, perspective_problem, voxel_type):
    from oracle import oracle as O
    from ettention_b200 import _abi
    from ettention_b200.operators import AlgebraicParameterSet
    geoms, projs = perspective_problem
    p = AlgebraicParameterSet(algorithm="blockIterative", block_size=8, iterations=2, lam=0.2,
                              order=_abi.ORDER_RANDOM, subvolume_count=2)
    v, order = cuda_recon(ctx, geoms, projs, PERSP_RES, p, 2, voxel_type=voxel_type, subvolumes=2)
    assert sorted(order) == list(range(len(geoms))) and order != list(range(len(geoms)))
    assert np.all(np.isfinite(v)) and np.abs(v).max() > 0
    if voxel_type == 0:
        vo = oracle_recon(geoms, projs, PERSP_RES, 0.2, 8, 2, order, 32, subvolumes=2)
        assert O.rel_l2(v, vo) <= RECON_TOL
    else:
        v64 = oracle_recon(geoms, projs, PERSP_RES, 0.2, 8, 2, order, 64, subvolumes=2)
        assert O.rel_l2(v, v64) <= BF16_TOL


PAR_RES = (128, 128, 32)


@pytest.fixture(scope="module")
def parallel_problem():
    from ettention_b200.operators import mrc_base_geometry
    from tests.helpers import ellipsoid_phantom
    res = PAR_RES
    phantom = ellipsoid_phantom(res, 40, axes=(4.0, 32.0), density=(0.0005, 0.01), seed=2002)
    geoms = [mrc_base_geometry(res[0], res[1]).rotated(float(a)) for a in np.linspace(-60.0, 60.0, 61)]
    return geoms, noisy_projections(phantom, geoms, res, 100.0, 2002)


@pytest.mark.parametrize("algo,block,iters,voxel_type", [("sirt", 0xFFFFFFFF, 4, 0), ("sirt", 0xFFFFFFFF, 4, 2),
                                                          ("sart", 1, 2, 2)])
def test_parallel_sirt_sart_storage(ctx, parallel_problem, algo, block, iters, voxel_type):
    from oracle import oracle as O
    from ettention_b200 import _abi
    from ettention_b200.operators import AlgebraicParameterSet
    geoms, projs = parallel_problem
    p = AlgebraicParameterSet(algorithm=algo, block_size=block, iterations=iters, lam=0.3 if algo == "sart" else 1.0,
                              order=_abi.ORDER_IDENTITY)
    v, order = cuda_recon(ctx, geoms, projs, PAR_RES, p, iters, voxel_type=voxel_type)
    assert order == list(range(61))
    nblock = 61 if algo == "sirt" else 1
    if voxel_type == 0:
        vo = oracle_recon(geoms, projs, PAR_RES, p.lam, nblock, iters, order, 32)
        assert O.rel_l2(v, vo) <= RECON_TOL
    else:
        v64 = oracle_recon(geoms, projs, PAR_RES, p.lam, nblock, iters, order, 64)
        assert O.rel_l2(v, v64) <= F16_TOL


def round_projections(projs, kind):
    """The tilt series as 16-bit storage keeps it: round to nearest even FP16 (numpy) or
    BF16 (the upper 16 bits after adding 0x7fff plus the kept bit's parity), widened back."""
    if kind == 1:
        return projs.astype(np.float16).astype(np.float32)
    bits = projs.astype(np.float32).view(np.uint32).astype(np.uint64)
    bits = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return bits.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("algo,fused", [("sart", "1"), ("sart", "0"), ("sirt", "1")])
def test_projection_storage_equals_prerounded_series(ctx, parallel_problem, kind, algo, fused, monkeypatch):
    """FP16 / BF16 storage of the tilt series: the reconstruction equals, bit for bit, the
    FP32-storage reconstruction of the series rounded to that format on the host -- on the
    fused persistent SART path, the unfused one, and SIRT -- with an FP16-shadow volume
    for SART (the C2 low-precision storage) and FP32 for SIRT."""
    from ettention_b200 import _abi
    from ettention_b200.operators import AlgebraicParameterSet, Context
    monkeypatch.setenv("ETCU_FUSED", fused)
    geoms, projs = parallel_problem
    vt = 2 if algo == "sart" else 0
    lam, block = (0.3, 1) if algo == "sart" else (1.0, 0xFFFFFFFF)
    c = Context(0)  # the environment is read when a context is created
    try:
        p16 = AlgebraicParameterSet(algorithm=algo, block_size=block, iterations=2, lam=lam,
                                    order=_abi.ORDER_IDENTITY, projection_storage=kind)
        v16, _ = cuda_recon(c, geoms, projs, PAR_RES, p16, 2, voxel_type=vt)
        p32 = AlgebraicParameterSet(algorithm=algo, block_size=block, iterations=2, lam=lam,
                                    order=_abi.ORDER_IDENTITY)
        vr, _ = cuda_recon(c, geoms, round_projections(projs, kind), PAR_RES, p32, 2, voxel_type=vt)
    finally:
        c.close()
    assert np.abs(v16).max() > 0
    assert np.array_equal(v16, vr)


@pytest.mark.parametrize("kind,tol", [(1, F16_TOL), (2, BF16_TOL)])
def test_projection_and_volume_16bit_storage_against_fp64_oracle(ctx, parallel_problem, kind, tol):
    """The C2 low-precision configuration: volume with a 16-bit shadow (FP16 or BF16) over
    an FP32 master and the tilt series stored in the same 16-bit format, SART, against the
    FP64 oracle on the FP32 series, at that format's storage bound."""
    from oracle import oracle as O
    from ettention_b200 import _abi
    from ettention_b200.operators import AlgebraicParameterSet
    geoms, projs = parallel_problem
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=_abi.ORDER_IDENTITY,
                              projection_storage=kind)
    v, order = cuda_recon(ctx, geoms, projs, PAR_RES, p, 2, voxel_type={1: 2, 2: 3}[kind])
    v64 = oracle_recon(geoms, projs, PAR_RES, 0.3, 1, 2, order, 64)
    assert O.rel_l2(v, v64) <= tol


def test_unknown_projection_storage_is_rejected(ctx, parallel_problem):
    from ettention_b200._abi import EttentionError
    from ettention_b200.operators import AlgebraicParameterSet
    geoms, projs = parallel_problem
    p = AlgebraicParameterSet(algorithm="sart", iterations=1, lam=0.3, projection_storage=7)
    with pytest.raises(EttentionError, match="unknown projection storage"):
        cuda_recon(ctx, geoms, projs, PAR_RES, p, 1)
