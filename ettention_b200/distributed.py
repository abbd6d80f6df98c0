"""One volume reconstructed on several GPUs: the reference's z-slab sub-volumes
(LR/model/volume/VolumeProperties.cpp:74-98) become one slab per rank.

Per block of the block-iterative loop (BlockIterativeReconstructionOperator.cpp:92-142):
every rank forward projects its slab for the block's views (partial line integrals
of volume and traversal length, which the reference already accumulates slab by slab
with `+=`, ParallelBeamsForwardProjection.cl:56-57), one all-reduce (sum) of the
block's (virtual, traversal) images makes them complete on every rank, every rank
forms the residual b - Ax (with long-object compensation when enabled), and each rank
back projects its own slab with lambda / blockSize.  The only data exchange is that
all-reduce: B x 2 x H x W floats per block.

`CudaSlabReconstruction` runs this on the GPU through the block-step C ABI
(etcu_recon_slab_forward / _step / _backward): the first block's forward projection of the
slab into a device buffer, then per block the NCCL all-reduce of its buffer enqueued on the
library's stream and one stream-ordered step -- its residual and back projection and the
next block's forward projection, for SART one fused step -- with no host synchronisation
inside an iteration.  `SlabDecomposedReconstruction` is the same loop
written against an engine (a rank's slab and its operators), which runs on CUDA
(`CudaSlabEngine`, operator by operator) and, in tests, on a CPU restatement with the gloo
backend.
"""
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _abi
from ._abi import EttentionError


def slab_split(resolution: Sequence[int], bbox_min: Sequence[float], bbox_max: Sequence[float],
               count: int) -> List[Tuple[int, int, List[float], List[float]]]:
    """z split of VolumeProperties.cpp:74-98 (remainder on the first slabs), in the
    float32 arithmetic of the library's sub-volume split: [(z0, rz, bmin, bmax)]."""
    X, Y, Z = (int(r) for r in resolution)
    if Z < count:
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT,
                             f"Volume of size {Z} in z direction cannot be split into {count} subvolumes!")
    f32 = np.float32
    lo = np.asarray(bbox_min, f32)
    hi = np.asarray(bbox_max, f32)
    vs = ((hi - lo) / np.asarray([X, Y, Z], f32)).astype(f32)
    base, rem = Z // count, Z - count * (Z // count)
    nxt = lo.copy()
    out, z0 = [], 0
    for i in range(count):
        rz = base + 1 if i < rem else base
        smax = (nxt + np.asarray([X, Y, rz], f32) * vs).astype(f32)
        out.append((z0, rz, [float(v) for v in nxt], [float(v) for v in smax]))
        nxt = nxt.copy()
        nxt[2] = smax[2]
        z0 += rz
    return out


class CudaSlabEngine:
    """This rank's slab on its GPU: a GPUMappedVolume with the slab's bounding box and
    the operator-level calls of the C ABI; the all-reduce goes through
    torch.distributed (NCCL) when a process group is initialised."""

    def __init__(self, ctx, resolution, bbox_min, bbox_max, rank: int, world: int, voxel_type: int = 0):
        import torch
        from .operators import GPUMappedVolume
        self.torch = torch
        self.ctx = ctx
        self.rank, self.world = rank, world
        z0, rz, lo, hi = slab_split(resolution, bbox_min, bbox_max, world)[rank]
        self.z0, self.rz = z0, rz
        self.full_bbox = (list(bbox_min), list(bbox_max))
        self.volume = GPUMappedVolume(ctx, (int(resolution[0]), int(resolution[1]), rz), lo, hi,
                                      voxel_type=voxel_type)
        self.device = torch.device("cuda", ctx.device)

    def zeros(self, shape):
        return self.torch.zeros(shape, dtype=self.torch.float32, device=self.device)

    def to_device(self, a: np.ndarray):
        return self.torch.as_tensor(np.ascontiguousarray(a, np.float32)).to(self.device)

    def upload(self, slab: np.ndarray) -> None:
        self.volume.upload(slab)

    def download(self) -> np.ndarray:
        return self.volume.download()

    def forward(self, geometry, samples: int, virtual, traversal) -> None:
        """Adds this slab's line integrals of volume and mask into virtual / traversal."""
        from .operators import ForwardProjectionOperator
        fp = ForwardProjectionOperator(self.volume, samples)
        fp.setScannerGeometry(geometry)
        fp.SetOutput(virtual, traversal)
        fp.Execute(0)

    def all_reduce(self, t) -> None:
        if self.world > 1:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.SUM)

    def residual(self, real, virtual, traversal, loc_length: Optional[float]):
        from .operators import compare, long_object_compensation
        if loc_length is not None:
            long_object_compensation(self.ctx, virtual, traversal, float(loc_length))
        res = self.torch.empty_like(virtual)
        compare(self.ctx, real, virtual, res)
        return res

    def back(self, geometry, residual, traversal, lam: float, block_size: int, samples: int, sampling: int) -> None:
        from .operators import BackProjectionOperator
        bp = BackProjectionOperator(self.volume, lam, samples, sampling)
        bp.setScannerGeometry(geometry)
        bp.setInput(residual, traversal, block_size)
        bp.execute()

    def close(self) -> None:
        self.volume.close()


class SlabDecomposedReconstruction:
    """BlockIterativeReconstructionOperator over z-slabs distributed across ranks.

    ``engine`` is this rank's slab (CudaSlabEngine or a CPU restatement with the same
    methods); ``projections`` is the (N, H, W) tilt series every rank holds; ``params``
    an AlgebraicParameterSet (block size, lambda, samples, order, long-object
    compensation, sampling)."""

    def __init__(self, engine, geometries, projections: np.ndarray, params):
        from .operators import projection_order
        self.engine = engine
        self.geometries = list(geometries)
        self.params = params
        n = len(self.geometries)
        self.order = projection_order(params.order, n, params.skip)
        if not self.order:
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "After applying SkipProjectionList no projections are left!")
        block = int(params.block_size)
        if block == 0:
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "Illegal ProjectionBlockSize!")
        self.block = min(block, len(self.order))
        self.real = engine.to_device(projections)
        self.H, self.W = int(projections.shape[1]), int(projections.shape[2])
        self.loc = None
        if params.use_long_object_compensation:  # traversal length of the complete volume
            lo, hi = engine.full_bbox
            self.loc = [g.traversal_length(lo, hi) for g in self.geometries]

    def runSingleIteration(self) -> None:
        p, e = self.params, self.engine
        M = len(self.order)
        fs = max(1, int(p.fp_samples))
        for first in range(0, M, self.block):
            ids = self.order[first:first + self.block]
            B = len(ids)
            buf = e.zeros((B, 2, self.H, self.W))  # (virtual, traversal) per view: one all-reduce
            for k, v in enumerate(ids):
                e.forward(self.geometries[v], fs, buf[k, 0], buf[k, 1])
            e.all_reduce(buf)
            res = [e.residual(self.real[v], buf[k, 0], buf[k, 1], None if self.loc is None else self.loc[v])
                   for k, v in enumerate(ids)]
            for k, v in enumerate(ids):  # BackProjectionKernel.cpp:94 lambda / blockSize
                e.back(self.geometries[v], res[k], buf[k, 1], float(p.lam), B, int(p.bp_samples), int(p.sampling))

    def runNiterations(self, n: int) -> None:
        for _ in range(int(n)):
            self.runSingleIteration()


class CudaSlabReconstruction:
    """This rank's z-slab of one volume, reconstructed with the block-step C ABI.

    Every rank holds the whole tilt series; rank r owns slab r of the reference's split.
    Block b's (B, 2, H, W) buffer receives the slab's line integrals and ray lengths of the
    block's views (etcu_recon_slab_forward for the first block, the previous step for the
    others), `torch.distributed.all_reduce` sums it over the ranks on the library's stream
    (NCCL when the process group uses it), and etcu_recon_slab_step forms b - Ax
    (long-object compensation over the complete volume), back projects the block into the
    slab with lambda / B and forward projects block b + 1 into the other buffer
    (etcu_recon_slab_backward for the last block)."""

    def __init__(self, ctx, resolution, bbox_min, bbox_max, rank: int, world: int, geometries,
                 projections: np.ndarray, params, voxel_type: int = 0):
        import ctypes
        import torch
        from .operators import BlockIterativeReconstructionOperator, GPUMappedVolume
        self.torch = torch
        self.ctx = ctx
        self.rank, self.world = rank, world
        z0, rz, lo, hi = slab_split(resolution, bbox_min, bbox_max, world)[rank]
        self.z0, self.rz = z0, rz
        self.volume = GPUMappedVolume(ctx, (int(resolution[0]), int(resolution[1]), rz), lo, hi, voxel_type=voxel_type)
        self.rec = BlockIterativeReconstructionOperator(self.volume, geometries, projections, params, use_graph=False)
        h = self.rec.handle
        bmin = (ctypes.c_float * 3)(*[float(v) for v in bbox_min])
        bmax = (ctypes.c_float * 3)(*[float(v) for v in bbox_max])
        ctx.check(_abi.lib().etcu_recon_set_complete_bbox(h, bmin, bmax))
        nb, bs = ctypes.c_uint32(), ctypes.c_uint32()
        ctx.check(_abi.lib().etcu_recon_block_count(h, ctypes.byref(nb), ctypes.byref(bs)))
        self.blocks, self.block_size = nb.value, bs.value
        self.views = len(self.rec.view_order())
        H, W = int(projections.shape[1]), int(projections.shape[2])
        dev = torch.device("cuda", ctx.device)
        # blocks alternate between two (B, 2, H, W) buffers: a step reads block b's complete
        # images while it writes block b + 1's partial ones
        self.bufs = [torch.zeros((self.block_size, 2, H, W), dtype=torch.float32, device=dev) for _ in range(2)]
        torch.cuda.synchronize(dev)
        self.stream = torch.cuda.ExternalStream(ctx.stream_handle)

    def block_views(self, b: int) -> int:
        return min(self.block_size, self.views - b * self.block_size)

    def buffer(self, b: int):
        """Block b's (virtual, traversal) images."""
        return self.bufs[b % 2]

    def block_forward(self, b: int) -> None:
        """This slab's partial images of block b into buffer(b)."""
        self.ctx.check(_abi.lib().etcu_recon_slab_forward(self.rec.handle, int(b), self.buffer(b).data_ptr()))

    def block_step(self, b: int) -> None:
        """Block b's residual and back projection (from the complete images in buffer(b)) and
        block b + 1's partial images into buffer(b + 1); one fused step for SART."""
        self.ctx.check(_abi.lib().etcu_recon_slab_step(self.rec.handle, int(b), self.buffer(b).data_ptr(),
                                                       self.buffer(b + 1).data_ptr()))

    def block_backward(self, b: int) -> None:
        """Residual from the complete images in buffer(b) and back projection into the slab."""
        self.ctx.check(_abi.lib().etcu_recon_slab_backward(self.rec.handle, int(b), self.buffer(b).data_ptr()))

    def all_reduce(self, b: int) -> None:
        if self.world > 1:
            import torch.distributed as dist
            with self.torch.cuda.stream(self.stream):
                dist.all_reduce(self.buffer(b)[:self.block_views(b)], op=dist.ReduceOp.SUM)

    def runSingleIteration(self) -> None:
        self.block_forward(0)
        for b in range(self.blocks):
            self.all_reduce(b)
            if b + 1 < self.blocks:
                self.block_step(b)
            else:
                self.block_backward(b)

    def runNiterations(self, n: int) -> None:
        for _ in range(int(n)):
            self.runSingleIteration()

    def last_residual_sq(self) -> float:
        return self.rec.last_residual_sq()

    def download(self) -> np.ndarray:
        return self.volume.download()

    def close(self) -> None:
        self.rec.close()
        self.volume.close()
