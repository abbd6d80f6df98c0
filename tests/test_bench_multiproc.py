"""Multi-process plumbing of bench.py at world size 2, on CPU with the gloo backend.

`bench.py --gpus N` runs one process per GPU, each reconstructing its own tilt series
(weak scaling; no collective on the data path).  The only collective is the timing:
every rank takes the max over ranks of its device time, in the same order on every
rank.  The reference arm runs on rank 0 only; the other ranks return without work.
"""
import io
import os
import socket
import contextlib

import pytest


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import bench
    try:
        r, w, local = bench.dist_init(timeout_s=60)
        m1 = bench.max_over_ranks(10.0 * r + 3.5, w)   # ranks disagree: the max wins
        bench.barrier(w)
        m2 = bench.max_over_ranks(1.25, w)             # ranks agree
        seed = bench.series_seed(r)

        class Args:
            steps = 1
            warmup = 0
        out = io.StringIO()
        ref_ran = True
        if r != 0:
            with contextlib.redirect_stdout(out):
                ref_ran = bench.run_reference(Args(), r, w) is not None or bool(out.getvalue())
        q.put((r, w, local, m1, m2, seed, ref_ran))
    except Exception as e:  # report to the parent instead of hanging it
        q.put(("error", rank, repr(e)))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_world2_timing_collective_seeds_and_reference_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    errors = [r for r in results if r[0] == "error"]
    assert not errors, errors
    results.sort()
    assert [r[0] for r in results] == [0, 1]
    assert all(r[1] == 2 and r[2] == r[0] for r in results)
    assert all(r[3] == 13.5 and r[4] == 1.25 for r in results)
    assert results[0][5] != results[1][5]          # every rank has its own series
    assert results[1][6] is False                  # the reference arm does nothing off rank 0
    assert all(p.exitcode == 0 for p in procs)


def test_single_process_needs_no_process_group(monkeypatch):
    import torch.distributed as dist
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_init() == (0, 1, 0)
    assert not dist.is_initialized()
    assert bench.max_over_ranks(7.0, 1) == 7.0


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_c4_series_are_dealt_out_once_and_evenly(world):
    """bench.py --workload c4 under torchrun: every one of the 64 independent series goes to
    exactly one rank, every rank computes the same deal, and the ranks' work (voxel-view
    updates per iteration) stays within the largest series of the mean."""
    import bench
    shapes = bench.c4_shapes()
    deal = [bench.c4_shard(shapes, r, world) for r in range(world)]
    flat = sorted(i for d in deal for i in d)
    assert flat == list(range(len(shapes)))
    assert deal == [bench.c4_shard(shapes, r, world) for r in range(world)]
    work = [s[0][0] * s[0][1] * s[0][2] * s[1] for s in shapes]
    loads = [sum(work[i] for i in d) for d in deal]
    assert max(loads) - min(loads) <= max(work)
