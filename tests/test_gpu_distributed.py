"""The z-slab decomposition driver (ettention_b200/distributed.py) with the CUDA engine at
world size 1: the per-view forward projection, residual (with long-object compensation)
and back projection through the operator-level C ABI must reproduce the single-GPU
reconstruction (BlockIterativeReconstructionOperator) for SART and SIRT.  Its
multi-rank behaviour is tested on CPU (tests/test_distributed_slabs.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("block,loc", [(1, False), (1, True), (9, True)])
def test_cuda_slab_engine_world1_equals_reconstruction(block, loc):
    from oracle import oracle as O
    from ettention_b200 import _abi
    from ettention_b200.distributed import CudaSlabEngine, SlabDecomposedReconstruction
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator, Context,
                                          GPUMappedVolume)
    from tests.test_distributed_slabs import X, Y, Z, problem
    geoms, projs = problem()
    p = AlgebraicParameterSet(algorithm="x", block_size=block, iterations=2, lam=0.3, order=_abi.ORDER_IDENTITY,
                              use_long_object_compensation=loc)
    ctx = Context(0)
    try:
        lo, hi = [-0.5 * X, -0.5 * Y, -0.5 * Z], [0.5 * X, 0.5 * Y, 0.5 * Z]
        eng = CudaSlabEngine(ctx, (X, Y, Z), lo, hi, rank=0, world=1)
        rec = SlabDecomposedReconstruction(eng, geoms, projs, p)
        rec.runNiterations(2)
        v = eng.download()
        eng.close()
        vol = GPUMappedVolume(ctx, (X, Y, Z))
        ref = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
        ref.runNiterations(2)
        r = ref.getReconstructedVolume()
        ref.close()
        vol.close()
    finally:
        ctx.close()
    assert np.abs(r).max() > 0
    assert O.rel_l2(v, r) <= 1e-6


def _params(block, loc, lam=0.3):
    from ettention_b200 import _abi
    from ettention_b200.operators import AlgebraicParameterSet
    return AlgebraicParameterSet(algorithm="x", block_size=block, iterations=2, lam=lam, order=_abi.ORDER_IDENTITY,
                                 use_long_object_compensation=loc)


@pytest.mark.parametrize("block,loc", [(1, False), (1, True), (4, True), (9, True)])
def test_block_step_abi_world1_equals_reconstruction(block, loc):
    """CudaSlabReconstruction (etcu_recon_slab_forward / _backward) with one rank against
    the single-GPU reconstruction: same volume and same data residual."""
    from oracle import oracle as O
    from ettention_b200.distributed import CudaSlabReconstruction
    from ettention_b200.operators import BlockIterativeReconstructionOperator, Context, GPUMappedVolume
    from tests.test_distributed_slabs import X, Y, Z, problem
    geoms, projs = problem()
    p = _params(block, loc)
    ctx = Context(0)
    try:
        lo, hi = [-0.5 * X, -0.5 * Y, -0.5 * Z], [0.5 * X, 0.5 * Y, 0.5 * Z]
        s = CudaSlabReconstruction(ctx, (X, Y, Z), lo, hi, 0, 1, geoms, projs, p)
        assert s.blocks == -(-N_VIEWS_ // min(block, N_VIEWS_))
        s.runNiterations(2)
        v, rs = s.download(), s.last_residual_sq()
        s.close()
        vol = GPUMappedVolume(ctx, (X, Y, Z))
        ref = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
        ref.runNiterations(2)
        r, rr = ref.getReconstructedVolume(), ref.last_residual_sq()
        ref.close()
        vol.close()
    finally:
        ctx.close()
    assert np.abs(r).max() > 0
    assert O.rel_l2(v, r) <= 1e-6
    assert abs(rs - rr) <= 1e-5 * rr


N_VIEWS_ = 9


@pytest.mark.parametrize("block,loc", [(1, True), (4, True), (9, False)])
def test_block_step_abi_two_slabs_equal_subvolume_reconstruction(block, loc):
    """Two ranks of the z-slab decomposition emulated in one process on one GPU: both
    slabs' partial images of a block are formed, summed (the all-reduce, done here by a
    plain add on the library's stream), then both slabs back project.  No kernel waits on
    another rank.  The assembled volume must equal the single-GPU reconstruction of a
    volume with two sub-volumes and the FP64 oracle's two-sub-volume reconstruction."""
    import torch
    from oracle import oracle as O
    from ettention_b200.distributed import CudaSlabReconstruction
    from ettention_b200.operators import BlockIterativeReconstructionOperator, Context, GPUMappedVolume
    from tests.helpers import oracle_geometry
    from tests.test_distributed_slabs import X, Y, Z, problem
    geoms, projs = problem()
    p = _params(block, loc)
    ctx = Context(0)
    try:
        lo, hi = [-0.5 * X, -0.5 * Y, -0.5 * Z], [0.5 * X, 0.5 * Y, 0.5 * Z]
        ranks = [CudaSlabReconstruction(ctx, (X, Y, Z), lo, hi, k, 2, geoms, projs, p) for k in range(2)]
        for it in range(2):
            for s in ranks:
                s.block_forward(0)
            for b in range(ranks[0].blocks):
                n = ranks[0].block_views(b)
                with torch.cuda.stream(ranks[0].stream):
                    tot = ranks[0].buffer(b)[:n] + ranks[1].buffer(b)[:n]
                    for s in ranks:
                        s.buffer(b)[:n].copy_(tot)
                for s in ranks:
                    if b + 1 < s.blocks and (it == 0 or b % 2):  # both the step and the split calls
                        s.block_step(b)
                    else:
                        s.block_backward(b)
                        if b + 1 < s.blocks:
                            s.block_forward(b + 1)
        ctx.synchronize()
        v = np.zeros((Z, Y, X), np.float32)
        for s in ranks:
            v[s.z0:s.z0 + s.rz] = s.download()
            s.close()
        vol = GPUMappedVolume(ctx, (X, Y, Z), subvolume_count=2)
        ref = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
        ref.runNiterations(2)
        r = ref.getReconstructedVolume()
        ref.close()
        vol.close()
    finally:
        ctx.close()
    vg = O.VolumeGeometry.centered((X, Y, Z), subvolumes=2)
    setup = O.ReconstructionSetup(vg, [oracle_geometry(g) for g in geoms], projs, 0.3, block, 1, 1, use_loc=loc)
    vo = np.zeros((Z, Y, X), np.float32)
    O.block_iterative(setup, vo, 2, 32)
    assert np.abs(r).max() > 0
    assert O.rel_l2(v, r) <= 1e-6
    assert O.rel_l2(v, vo) <= 1e-5
