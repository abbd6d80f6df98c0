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
