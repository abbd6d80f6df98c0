"""One volume over several ranks by z-slabs (ettention_b200/distributed.py), on CPU with
the gloo backend at world size 2: each rank runs the CPU restatement of the kernels on
its slab (an engine with the same methods as CudaSlabEngine), the block's virtual and
traversal images are summed by one all-reduce, every rank forms the residual, each
back projects its slab.  The volume assembled from the ranks must equal the
single-process oracle reconstruction with two sub-volumes, for SART, SIRT and block
size 4, with long-object compensation."""
import os
import socket

import numpy as np
import pytest

X, Y, Z = 40, 24, 18
N_VIEWS = 9


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class OracleSlabEngine:
    """The CPU restatement of forward / back projection on this rank's slab."""

    def __init__(self, resolution, rank, world):
        import torch
        from oracle import oracle as O
        from ettention_b200.distributed import slab_split
        self.torch, self.O = torch, O
        self.rank, self.world = rank, world
        self.vg = O.VolumeGeometry.centered(resolution)
        z0, rz, lo, hi = slab_split(resolution, self.vg.bmin, self.vg.bmax, world)[rank]
        self.z0, self.rz = z0, rz
        self.slab = dict(res=(resolution[0], resolution[1], rz), z0=z0, bmin=np.float32(lo), bmax=np.float32(hi))
        self.full_bbox = (list(self.vg.bmin), list(self.vg.bmax))
        self.vol = np.zeros((rz, resolution[1], resolution[0]), np.float32)

    def zeros(self, shape):
        return self.torch.zeros(shape, dtype=self.torch.float32)

    def to_device(self, a):
        return self.torch.as_tensor(np.ascontiguousarray(a, np.float32))

    def forward(self, geometry, samples, virtual, traversal):
        from tests.helpers import oracle_geometry
        self.O.forward_project(self.vol, self.vg, oracle_geometry(geometry), samples, 32, slab=self.slab,
                               proj=virtual.numpy(), length=traversal.numpy())

    def all_reduce(self, t):
        import torch.distributed as dist
        if self.world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)

    def residual(self, real, virtual, traversal, loc_length):
        v, l = virtual.numpy(), traversal.numpy()
        if loc_length is not None:
            pv, pl = self.O.long_object_compensation(v, l, loc_length)
            v[...] = pv
            l[...] = pl
        return self.torch.as_tensor((real.numpy() - v).astype(np.float32))

    def back(self, geometry, residual, traversal, lam, block_size, samples, sampling):
        from tests.helpers import oracle_geometry
        self.O.back_project(self.vol, self.vg, oracle_geometry(geometry), residual.numpy(), traversal.numpy(),
                            np.float32(lam) / np.float32(block_size), samples, 32,
                            self.O.WEIGHTS_EXACT if sampling == 1 else self.O.WEIGHTS_Q8, slab=self.slab)


def problem():
    from oracle import oracle as O
    from ettention_b200.operators import mrc_base_geometry
    from tests.helpers import ellipsoid_phantom, oracle_geometry
    truth = ellipsoid_phantom((X, Y, Z), 5, seed=77)
    geoms = [mrc_base_geometry(X, Y).rotated(float(a)) for a in np.linspace(-60, 60, N_VIEWS)]
    vg = O.VolumeGeometry.centered((X, Y, Z))
    projs = np.stack([O.forward_project(truth, vg, oracle_geometry(g), 1, 32)[0] for g in geoms])
    return geoms, projs.astype(np.float32)


def _worker(rank, world, port, block, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        from ettention_b200 import _abi
        from ettention_b200.distributed import SlabDecomposedReconstruction
        from ettention_b200.operators import AlgebraicParameterSet
        geoms, projs = problem()
        p = AlgebraicParameterSet(algorithm="x", block_size=block, iterations=2, lam=0.3,
                                  order=_abi.ORDER_IDENTITY, use_long_object_compensation=True)
        eng = OracleSlabEngine((X, Y, Z), rank, world)
        rec = SlabDecomposedReconstruction(eng, geoms, projs, p)
        rec.runNiterations(2)
        q.put((rank, eng.z0, eng.vol.copy()))
    except Exception as e:
        q.put(("error", rank, repr(e)))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


@pytest.mark.parametrize("block", [1, N_VIEWS, 4])
def test_two_rank_slab_decomposition_equals_oracle(block):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    from tests.helpers import oracle_geometry
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, block, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    errors = [r for r in results if r[0] == "error"]
    assert not errors, errors
    vol = np.zeros((Z, Y, X), np.float32)
    for rank, z0, slab in results:
        vol[z0:z0 + slab.shape[0]] = slab
    geoms, projs = problem()
    vg = O.VolumeGeometry.centered((X, Y, Z), subvolumes=2)
    setup = O.ReconstructionSetup(vg, [oracle_geometry(g) for g in geoms], projs, 0.3, block, 1, 1, use_loc=True)
    vo = np.zeros((Z, Y, X), np.float32)
    O.block_iterative(setup, vo, 2, 32)
    assert O.rel_l2(vol, vo) <= 1e-6
    assert np.abs(vo).max() > 0


def test_slab_split_matches_the_library_rule():
    from oracle import oracle as O
    from ettention_b200.distributed import slab_split
    vg = O.VolumeGeometry.centered((50, 30, 23), dimension=(64.0, 40.0, 29.5), subvolumes=4)
    ref = vg.slabs()
    got = slab_split(vg.resolution, vg.bmin, vg.bmax, 4)
    assert [(g[0], g[1]) for g in got] == [(s["z0"], s["res"][2]) for s in ref]
    for g, s in zip(got, ref):
        assert np.array_equal(np.float32(g[2]), s["bmin"]) and np.array_equal(np.float32(g[3]), s["bmax"])
