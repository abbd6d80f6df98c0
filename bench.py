#!/usr/bin/env python
"""Benchmark of the B200 block-iterative reconstruction path.

Workload (one "step" = one full SART iteration over the tilt series):
  volume 1024 x 1024 x 256 float32, ellipsoid phantom (200 ellipsoids, semi-axes
  8-128 voxels, densities 0.05-1.0, scaled by 0.01 per voxel so line integrals
  stay in the range where 100-count Poisson noise is informative);
  61 parallel-beam views -60..+60 deg step 2, detector 1024 x 1024, pitch 1;
  Poisson noise at 100 counts/pixel then -log; SART (block 1), lambda 0.3,
  identity order, zero initial volume.  Synthetic data, seeded per rank.

  metric  "SART s to reach plain 30-iter residual": the plain-SART time to
          run 30 iterations = 30 x measured seconds per iteration (lower is better).
  value   device-resident inputs (projections and volume in HBM), one CUDA
          graph per iteration, CUDA events on the library stream, max over ranks.
  e2e     the same metric through the one-call C ABI etcu_reconstruct with host
          buffers: pinned host projections + volume in, 30 iterations, volume out.

Multi-GPU: one process per GPU, each reconstructs its own independent tilt
series (weak scaling); the only collective is the timing max over ranks.
`--impl reference` times the CPU restatement of the reference's kernels
(the reference's OpenCL build cannot run here) on a bounded sample.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_VIEWS = 61
RES = (1024, 1024, 256)  # x, y, z
DET = (1024, 1024)
LAMBDA = 0.3
I0 = 100.0
MU_SCALE = 0.01
TARGET_ITERS = 30
WORKLOAD = "SART parallel beam, 1024x1024x256 f32 volume, 61 views +-60 deg step 2, 1024^2 detector, Poisson I0=100"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-reps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--c4-f32", action="store_true", help="--workload c4 with FP32 volumes (default: FP16 shadow)")
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"],
                    help="headline workload's storage: f32, or an FP32 master volume with an FP16 / BF16 shadow and "
                         "the tilt series stored in the same 16-bit format")
    ap.add_argument("--no-autotune", action="store_true", help="built-in launch shapes instead of the autotuner's")
    ap.add_argument("--no-c5", action="store_true",
                    help="leave out the learned-warm-start (C5) record that the default 1-GPU run adds to its line")
    ap.add_argument("--no-c3", action="store_true",
                    help="leave out the perspective (C3) record that the default 1-GPU run adds to its line")
    ap.add_argument("--c5-seeds", type=int, default=100, help="held-out series of --workload c5")
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c4", "c5", "blobs", "slabs"],
                    help="c2: the headline SART workload (default); c3: 2048^2 x 512 perspective, block 8, "
                         "bf16 shadow; c4: 64 batched series of uneven sizes; slabs: the c2 volume split "
                         "into z-slabs over the ranks (strong scaling)")
    ap.add_argument("--c3-res", default="2048,2048,512",
                    help="volume (x,y,z) of --workload c3; the detector is x by y (smaller cases for ncu captures)")
    ap.add_argument("--ncu-case", action="store_true",
                    help="small profiling case for ncu: 512x512x256 volume, 8 views, one SART iteration "
                         "launched kernel by kernel, then per-kernel times of the unfused kernels")
    ap.add_argument("--warmstart-case", action="store_true",
                    help="profiling case of the learned warm start: three inferences of the trained network on a "
                         "256x256x128 volume (one 3-iteration SART volume of a held-out series)")
    ap.add_argument("--ncu-res", default="512,512,256",
                    help="volume of the --ncu-case (x,y,z; the detector is x by y)")
    return ap.parse_args()


# ------------------------------------------------------------------ distributed plumbing
_DIST_DEVICE = "cpu"


def dist_init(timeout_s: int = 300):
    """One process per GPU (torchrun env).  NCCL when CUDA is present, else gloo on CPU
    (the multi-process logic is tested that way).  Returns (rank, world, local rank)."""
    global _DIST_DEVICE
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                    device_id=torch.device("cuda", local))
            _DIST_DEVICE = "cuda"
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
            _DIST_DEVICE = "cpu"
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_DIST_DEVICE)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def series_seed(rank: int) -> int:
    """Each rank reconstructs its own tilt series (weak scaling, no data-path collective)."""
    return 2000 + rank


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        cmd = ["nvidia-smi", "-i", str(self.device),
               "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.lines:
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ workload
def make_phantom_torch(seed: int, device, res=None, count: int = 200, axes=(8.0, 128.0)):
    """`count` ellipsoids (centres uniform, semi-axes U(axes), uniform rotation,
    density U(0.05,1.0), additive), scaled by MU_SCALE; built on the GPU."""
    from ettention_b200.phantom import ellipsoid_phantom
    return ellipsoid_phantom(seed, device, RES if res is None else res, count, axes, mu_scale=MU_SCALE)


def make_problem(ctx, seed: int, keep_phantom: bool = False):
    """Phantom, tilt geometry and noisy projections (forward projected by the CUDA path);
    with keep_phantom also a host copy of the phantom."""
    import torch
    from ettention_b200.operators import ForwardProjectionOperator, GPUMappedVolume, mrc_base_geometry
    dev = torch.device("cuda", ctx.device)
    phantom = make_phantom_torch(seed, dev)
    torch.cuda.synchronize(dev)
    angles = np.linspace(-60.0, 60.0, N_VIEWS)
    geoms = [mrc_base_geometry(*DET).rotated(float(a)) for a in angles]
    vol = GPUMappedVolume(ctx, RES)
    host_phantom = phantom.cpu().numpy()
    vol.upload(host_phantom)
    del phantom
    fp = ForwardProjectionOperator(vol, 1)
    projs = torch.zeros((N_VIEWS, DET[1], DET[0]), dtype=torch.float32, device=dev)
    scratch = torch.zeros((DET[1], DET[0]), dtype=torch.float32, device=dev)
    for i, g in enumerate(geoms):
        fp.setScannerGeometry(g)
        fp.SetOutput(projs[i], scratch)
        fp.Execute(0)
    vol.close()
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    counts = torch.poisson(I0 * torch.exp(-projs), generator=gen)
    b = -torch.log(torch.clamp(counts, min=1.0) / I0)
    torch.cuda.synchronize(dev)
    if keep_phantom:
        return geoms, b.contiguous(), host_phantom
    return geoms, b.contiguous()


# ------------------------------------------------------------------ byte model
def algorithmic_bytes():
    """Per launch, FP32 storage, by the per-unit byte model (one forward-projection view:
    the volume read once, b read, (r, L) written; one back-projection view of a one-view
    block: the volume read and written once, (r, L) read).  A fused SART step processes
    one unit of each, so its algorithmic bytes are their sum."""
    V = RES[0] * RES[1] * RES[2]
    P = DET[0] * DET[1]
    fp = V * 4 + P * 4 + P * 8
    bp = 2 * V * 4 + P * 8
    return fp, bp, fp + bp


def fused_moved_bytes():
    """Bytes the fused step must move: the volume read and written once, view p's (r, L)
    read, view p + 1's b read and (r, L) written."""
    V = RES[0] * RES[1] * RES[2]
    P = DET[0] * DET[1]
    return 2 * V * 4 + P * 8 + P * 4 + P * 8


def source_key() -> str:
    """Hash of the CUDA source that defines the reconstruction kernels: a DRAM-traffic
    figure recorded from an ncu capture is used only while the kernels are built from the
    same source."""
    import hashlib
    h = hashlib.sha256()
    with open(os.path.join(ROOT, "ettention_b200", "csrc", "kernels.cuh"), "rb") as fh:
        h.update(fh.read())
    return h.hexdigest()[:16]


def recorded_traffic(kernel: str):
    """DRAM bytes per unit (`dram__bytes_read.sum + dram__bytes_write.sum` of one ncu
    capture, per voxel of one step) recorded in a profile summary as
    `traffic-key: <kernel> <source key> <bytes per voxel per step> <case>`, or None when no
    summary matches this build's sources."""
    key = source_key()
    pdir = os.path.join(ROOT, "profiles")
    for f in sorted(os.listdir(pdir)) if os.path.isdir(pdir) else ():
        if not f.endswith(".md"):
            continue
        for ln in open(os.path.join(pdir, f)):
            parts = ln.strip().strip("`").split()
            if len(parts) >= 5 and parts[0] == "traffic-key:" and parts[1] == kernel and parts[2] == key:
                return float(parts[3]), f"{f}: ncu capture of {parts[4]}"
    return None


def work_units(geoms):
    """Algorithmic work of one iteration in two units: forward-projection ray-voxel
    steps (every ray of every view counted from the voxels it enters and leaves the volume
    in: 1 + x cells crossed + z cells crossed; the views are tilted about y, so every
    detector row repeats its rays' xz path) and back-projection voxel-view updates."""
    X, Y, Z = RES
    lo = np.array([-0.5 * X, -0.5 * Y, -0.5 * Z])
    hi = -lo
    steps = 0
    for g in geoms:
        src, det = np.asarray(g.source, np.float64), np.asarray(g.detector, np.float64)
        hp, vp = np.asarray(g.hpitch, np.float64), np.asarray(g.vpitch, np.float64)
        d = det - src
        d /= np.linalg.norm(d)
        i = np.arange(g.width, dtype=np.float64) + 0.5
        o = src[None, :] + i[:, None] * hp[None, :] + (0.5 * g.height) * vp[None, :]
        with np.errstate(divide="ignore", invalid="ignore"):
            t0 = np.where(d != 0, (lo - o) / d, -np.inf)
            t1 = np.where(d != 0, (hi - o) / d, np.inf)
        tin = np.max(np.minimum(t0, t1), axis=1)
        tout = np.min(np.maximum(t0, t1), axis=1)
        hit = tout > tin
        pin = o + tin[:, None] * d
        pout = o + tout[:, None] * d
        cin = np.clip(np.floor(pin - lo), 0, np.array(RES) - 1)
        cout = np.clip(np.floor(pout - lo - 1e-9 * np.sign(d)), 0, np.array(RES) - 1)
        n = 1 + np.abs(cout[:, 0] - cin[:, 0]) + np.abs(cout[:, 2] - cin[:, 2])
        steps += int(n[hit].sum()) * g.height
    return steps, X * Y * Z * len(geoms)


# ------------------------------------------------------------------ CPU baseline (oracle)
CPU_SAMPLE_VIEWS = (0, 15, 30, 45, 60)  # -60, -30, 0, +30, +60 degrees of the 61-view series


def cpu_sample_problem(phantom):
    """The CPU sample's inputs: the views CPU_SAMPLE_VIEWS of the bench series and their
    noisy projections (the oracle's line integrals of the phantom, Poisson at I0, -log),
    made before the timed region."""
    from oracle import oracle as O
    vg = O.VolumeGeometry.centered(RES)
    base = O.mrc_base_geometry(*DET)
    angles = np.linspace(-60.0, 60.0, N_VIEWS)
    rng = np.random.Generator(np.random.PCG64(7))
    geoms, bs = [], []
    for i in CPU_SAMPLE_VIEWS:
        g = O.rotate_geometry(base, float(angles[i]))
        p, _ = O.forward_project(phantom, vg, g, 1, 32)
        counts = rng.poisson(I0 * np.exp(-p.astype(np.float64)))
        geoms.append(g)
        bs.append((-np.log(np.maximum(counts, 1) / I0)).astype(np.float32))
    return vg, geoms, bs


def cpu_sample_seconds(problem, threads: int):
    """Seconds per SART view of the FP32 CPU restatement of the reference kernels (oracle/)
    on `threads` host threads: forward projection, residual and back projection (texture
    weights rounded to 1/256, the mode the GPU path runs) of the sampled views, in order,
    from a zero volume as the first iteration starts."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    vg, geoms, bs = problem
    X, Y, Z = RES
    vol = np.zeros((Z, Y, X), np.float32)
    t0 = time.perf_counter()
    for g, b in zip(geoms, bs):
        p, l = O.forward_project(vol, vg, g, 1, 32)
        r = b - p
        O.back_project(vol, vg, g, r, l, LAMBDA, 1, 32, O.WEIGHTS_Q8)
    return (time.perf_counter() - t0) / len(geoms)


CPU_SAMPLE_TEXT = ("5 of the 61 views (-60, -30, 0, +30, +60 deg; FP + residual + Q8 BP each) at full size on "
                   "the bench phantom, FP32 oracle; seconds per view x61 views x30 iterations")


def run_reference(args, rank, world):
    """Reference arm: the CPU restatement of the reference's path on all host cores."""
    if rank != 0:
        return
    import torch
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    phantom = make_phantom_torch(series_seed(0), "cpu").numpy()
    problem = cpu_sample_problem(phantom)
    del phantom
    for _ in range(args.warmup):
        cpu_sample_seconds(problem, threads)
    ts = [cpu_sample_seconds(problem, threads) for _ in range(args.steps)]
    per_view = statistics.mean(ts)
    value = per_view * N_VIEWS * TARGET_ITERS
    line = {"impl": "reference", "metric": "SART s to reach plain 30-iter residual", "value": value, "unit": "s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": per_view * len(CPU_SAMPLE_VIEWS) * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": WORKLOAD, "step": "5 sampled views of one SART iteration",
                                            "host_threads": threads},
            "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port", "sample": CPU_SAMPLE_TEXT},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's OpenCL build cannot be compiled or run on this box; this arm times the "
                    "FP32 CPU restatement of its kernels (oracle/) on all host threads"}
    print(json.dumps(line), flush=True)


def run_e2e(args, ctx, geoms, b, params, world, lib_stream, vol_type=0):
    """30 iterations through etcu_reconstruct with pinned host buffers (in and out)."""
    import torch
    from ettention_b200 import _abi
    from ettention_b200._abi import View, VolumeDesc, lib
    host_proj = torch.empty(b.shape, dtype=torch.float32, pin_memory=True)
    host_proj.copy_(b.cpu())
    X, Y, Z = RES
    host_vol = torch.zeros((Z, Y, X), dtype=torch.float32, pin_memory=True)
    views = (View * N_VIEWS)(*[g.to_view() for g in geoms])
    desc = VolumeDesc()
    for i in range(3):
        desc.resolution[i] = RES[i]
        desc.bbox_min[i] = -0.5 * RES[i]
        desc.bbox_max[i] = 0.5 * RES[i]
    desc.subvolume_count = 1
    rp = params.recon_params(True)
    torch.cuda.empty_cache()
    e2e_times = []
    for rep in range(1 + args.e2e_reps):
        host_vol.zero_()
        barrier(world)
        ctx.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lib_stream)
        ctx.check(lib().etcu_reconstruct(ctx.handle, ctypes.byref(desc), vol_type, views, N_VIEWS,
                                         host_proj.data_ptr(), ctypes.byref(rp), TARGET_ITERS, host_vol.data_ptr()))
        e1.record(lib_stream)
        torch.cuda.synchronize()
        if rep > 0:
            e2e_times.append(e0.elapsed_time(e1))
    e2e_ms = max_over_ranks(statistics.mean(e2e_times), world)
    h2d = host_proj.numel() * 4 + host_vol.numel() * 4
    d2h = host_vol.numel() * 4
    # the host link's own speed on this box, for reading the e2e figure: one pinned copy
    # of the volume each way
    dev_vol = torch.empty(host_vol.shape, dtype=torch.float32, device="cuda")
    c0, c1, c2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    c0.record()
    dev_vol.copy_(host_vol, non_blocking=True)
    c1.record()
    host_vol.copy_(dev_vol, non_blocking=True)
    c2.record()
    c2.synchronize()
    link = {"h2d_gbs": host_vol.numel() * 4 / (c0.elapsed_time(c1) * 1e-3) / 1e9,
            "d2h_gbs": host_vol.numel() * 4 / (c1.elapsed_time(c2) * 1e-3) / 1e9}
    del dev_vol
    return {"value": e2e_ms * 1e-3, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "host_link": link}


# ------------------------------------------------------------------ ours
def run_ours(args, rank, world, local):
    import torch
    from ettention_b200 import _abi
    from ettention_b200._abi import ReconParams, View, VolumeDesc, check, lib
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator, Context,
                                          GPUMappedVolume)
    torch.cuda.set_device(local)
    ctx = Context(local)
    geoms, b, phantom = make_problem(ctx, series_seed(rank), keep_phantom=True)
    cpu_problem = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_problem = cpu_sample_problem(phantom)
    del phantom
    vt, ps = {"f32": (_abi.VOXEL_FLOAT32, _abi.PROJ_F32), "f16": (_abi.VOXEL_F16_MASTER, _abi.PROJ_F16),
              "bf16": (_abi.VOXEL_BF16_MASTER, _abi.PROJ_BF16)}[args.storage]
    params = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=TARGET_ITERS, lam=LAMBDA,
                                   order=_abi.ORDER_IDENTITY, projection_storage=ps)
    vol = GPUMappedVolume(ctx, RES, voxel_type=vt)
    rec = BlockIterativeReconstructionOperator(vol, geoms, b, params, use_graph=True)
    launches_per_iter = rec.launches_per_iteration
    d0 = rec.data_residual_sq()
    for _ in range(args.warmup):
        rec.runNiterations(1)
    ctx.synchronize()
    # ---- timed region: K iterations, CUDA events on the library stream ----
    cudart = torch.cuda.cudart()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    lib_stream = torch.cuda.ExternalStream(ctx.stream_handle)  # events on the stream the kernels run on
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ev0.record(lib_stream)
        rec.runNiterations(args.steps)
        ev1.record(lib_stream)
        ctx.synchronize()
        torch.cuda.synchronize()
    barrier(world)
    ms_total = ev0.elapsed_time(ev1)
    ms_total = max_over_ranks(ms_total, world)
    ms_per_step = ms_total / args.steps
    value = TARGET_ITERS * ms_per_step / 1e3
    d1 = rec.data_residual_sq()
    # ---- per-step device times (one more real iteration, issued as run() issues it,
    # CUDA events around every step on the library stream) ----
    steps = rec.profile_steps()
    fp_bytes, bp_bytes, fused_bytes = algorithmic_bytes()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    V = RES[0] * RES[1] * RES[2]
    per_kernel = {}
    # the persistent fused kernel runs all N_VIEWS - 1 fused steps of an iteration in one
    # launch; the per-step kernel one step per launch
    fused_launches = sum(l for k, _, l in steps if k == "fused")
    pairs = (N_VIEWS - 1) // fused_launches if fused_launches else 1
    fused_bytes *= pairs
    kernels = {"fused": "sart_fused_persistent_kernel" if pairs > 1 else "sart_fused_kernel",
               "forward": "forward_project_kernel", "back": "bp_sart_column_kernel"}
    for kind, name, byts, units in (("fused", "sart_fused_step", fused_bytes, pairs),
                                    ("forward", "forward_project", fp_bytes, 1),
                                    ("back", "back_project", bp_bytes, 1)):
        ts = [t for k, t, _ in steps if k == kind]
        if not ts:
            continue
        avg = sum(ts) / len(ts)
        gbs = byts / (avg * 1e-3) / 1e9
        rec_t = recorded_traffic(kernels[kind])
        per_kernel[name] = {"kernel": kernels[kind], "avg_ms": avg,
                            "launches": sum(l for k, _, l in steps if k == kind),
                            "total_ms": sum(ts), "algorithmic_bytes": byts, "gbs": gbs, "frac": gbs / hbm_peak,
                            "traffic": rec_t[0] * V * units if rec_t else None,
                            "traffic_source": rec_t[1] if rec_t else "no ncu capture recorded for this build"}
    if "sart_fused_step" in per_kernel:
        fk = per_kernel["sart_fused_step"]
        moved = fused_moved_bytes() * pairs
        fk["view_pairs_per_launch"] = pairs
        fk["moved_bytes"] = moved
        fk["moved_gbs"] = moved / (fk["avg_ms"] * 1e-3) / 1e9
        fk["moved_frac"] = fk["moved_gbs"] / hbm_peak
    dominant = max(per_kernel, key=lambda n: per_kernel[n]["total_ms"])
    dk = per_kernel[dominant]
    roofline = {"bound": "hbm", "kernel": dk["kernel"], "achieved": dk["gbs"], "peak": hbm_peak, "unit": "GB/s",
                "frac": dk["frac"], "peak_source": peak_src, "traffic": dk["traffic"],
                "bytes_model": ("one forward-projection view + one back-projection view per fused step "
                                "(4V+4P+8P + 8V+8P) x view_pairs_per_launch; the launch moves moved_bytes of them"
                                if dominant == "sart_fused_step" else "per-view byte model"),
                "traffic_source": dk["traffic_source"], "source_key": source_key(),
                "per_kernel": per_kernel}
    rec.close()
    vol.close()
    # ---- e2e: one-call host-buffer reconstruction through the C ABI ----
    e2e = None
    if args.e2e_reps > 0:
        e2e = run_e2e(args, ctx, geoms, b, params, world, lib_stream, vt)
    del b
    # ---- CPU baseline (rank 0, N = 1 only) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t = cpu_sample_seconds(cpu_problem, threads)
        cpu = {"value": t * N_VIEWS * TARGET_ITERS, "unit": "s", "cores": threads, "kind": "port",
               "sample": CPU_SAMPLE_TEXT}
    # ---- the perspective workload's record (1 GPU only): its own clocks, roofline and
    # CPU sample, in the same line ----
    ctx.close()
    # ---- the learned warm start against plain SART (1 GPU only): 20 held-out series ----
    c5 = None
    if rank == 0 and world == 1 and not args.no_c5:
        torch.cuda.empty_cache()
        try:
            c5 = run_c5(argparse.Namespace(**{**vars(args), "c5_seeds": min(args.c5_seeds, 20), "warmup": 3}))
            c5.pop("per_seed", None)
        except Exception as exc:  # the headline line is printed either way
            c5 = {"error": f"{type(exc).__name__}: {exc}"}
    c3 = None
    if rank == 0 and world == 1 and not args.no_c3:
        torch.cuda.empty_cache()
        try:
            c3 = run_c3(args, steps=3, warmup=3, cpu_baseline=not args.no_cpu_baseline)
        except Exception as exc:  # the headline line is printed either way
            c3 = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0:
        fp_steps, bp_updates = work_units(geoms)
        line = {"metric": "SART s to reach plain 30-iter residual", "value": value, "unit": "s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded ellipsoid phantom, CUDA-forward-projected, Poisson noise)",
                "config": {"workload": WORKLOAD, "step": "one SART iteration (61 views, one CUDA graph)",
                           "volume": list(RES), "views": N_VIEWS, "detector": list(DET), "lambda": LAMBDA,
                           "storage": args.storage if args.storage == "f32" else
                           f"f32 master + {args.storage} shadow, {args.storage} tilt series",
                           "l2": "inputs larger than L2 (1 GiB volume)",
                           "parallelism": f"independent series per GPU x{world}"},
                "e2e": e2e,
                "gpu_launches": launches_per_iter * args.steps,
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks.summary(),
                "work": {"fp_ray_voxel_steps": fp_steps, "bp_voxel_view_updates": bp_updates,
                         "units_per_s": (fp_steps + bp_updates) / (ms_per_step * 1e-3),
                         "fp_steps_source": "entry and exit voxels of every ray of the 61 views"},
                "residual_sq": {"before": d0, "after_warmup_and_timed": d1},
                "c3": c3,
                "c5": c5}
        print(json.dumps(line), flush=True)


def run_slabs(args, rank, world, local):
    """One volume over the ranks by z-slabs (strong scaling): the headline workload's
    volume split as the library splits sub-volumes, every rank holding the whole tilt
    series; per view, the slab's forward projection (etcu_recon_slab_forward), one
    all-reduce of the (virtual, traversal) images on the library's stream (NCCL, world > 1),
    the residual and the slab's back projection (etcu_recon_slab_backward)."""
    import torch
    from ettention_b200 import _abi
    from ettention_b200.distributed import CudaSlabReconstruction
    from ettention_b200.operators import AlgebraicParameterSet, Context
    torch.cuda.set_device(local)
    ctx = Context(local)
    geoms, b = make_problem(ctx, series_seed(0))
    params = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=TARGET_ITERS, lam=LAMBDA,
                                   order=_abi.ORDER_IDENTITY)
    lo = [-0.5 * r for r in RES]
    hi = [0.5 * r for r in RES]
    rec = CudaSlabReconstruction(ctx, RES, lo, hi, rank, world, geoms, b, params)
    for _ in range(args.warmup):
        rec.runSingleIteration()
    ctx.synchronize()
    stream = rec.stream
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        rec.runNiterations(args.steps)
        ev1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
    barrier(world)
    ms_per_step = max_over_ranks(ev0.elapsed_time(ev1), world) / args.steps
    rsq = rec.last_residual_sq()
    slab = [rec.z0, rec.rz]
    rec.close()
    ctx.close()
    if rank == 0:
        P = DET[0] * DET[1]
        print(json.dumps({
            "metric": "SART s to reach plain 30-iter residual", "value": TARGET_ITERS * ms_per_step / 1e3,
            "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ellipsoid phantom, CUDA-forward-projected, Poisson noise)",
            "config": {"workload": WORKLOAD, "step": "one SART iteration, block-step C ABI per view",
                       "parallelism": f"z-slabs x{world}", "slab_of_rank0": slab,
                       "all_reduce_bytes_per_view": 2 * P * 4 if world > 1 else 0,
                       "l2": "inputs larger than L2 (1 GiB volume)"},
            "gpu_launches": 3 * N_VIEWS * args.steps,  # per view: slab forward, residual, back projection
            "residual_sq_last_iteration": rsq, "clocks": clocks.summary()}), flush=True)


def run_ncu_case(res=(512, 512, 256)):
    """A case small enough for an ncu capture (by default a 256 MB volume, larger than L2)."""
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator, Context,
                                          GPUMappedVolume, mrc_base_geometry)
    X, Y, Z = res
    ctx = Context(0)
    rng = np.random.Generator(np.random.PCG64(0))
    vol = GPUMappedVolume(ctx, (X, Y, Z))
    vol.upload(rng.uniform(0, 0.01, (Z, Y, X)).astype(np.float32))
    geoms = [mrc_base_geometry(X, Y).rotated(float(a)) for a in np.linspace(-60, 60, 8)]
    projs = rng.uniform(0, 3, (8, Y, X)).astype(np.float32)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=1, lam=LAMBDA, order=_abi.ORDER_IDENTITY)
    rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p, use_graph=False)
    rec.runNiterations(1)
    f, b, nf, nb = rec.profile_iteration()
    print(json.dumps({"ncu_case": f"{X}x{Y}x{Z} f32, 8 views, SART", "forward_ms": f / nf, "back_ms": b / nb}))
    rec.close()
    vol.close()
    ctx.close()


# ------------------------------------------------------------------ C4: many uneven series
C4_SERIES = 64


def c4_shapes(seed: int = 4000):
    """64 seeded tilt series between 96^3 and 256x256x128 voxels, 41 to 81 views over
    +-50 to +-70 degrees (detector = volume x by y, pitch 1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(C4_SERIES):
        X = int(rng.integers(6, 17)) * 16
        Y = int(rng.integers(6, 17)) * 16
        Z = int(rng.integers(6, 9)) * 16
        nv = int(rng.integers(20, 41)) * 2 + 1
        tmax = float(rng.uniform(50.0, 70.0))
        out.append(((X, Y, Z), nv, tmax))
    return out


def c4_shard(shapes, rank: int, world: int):
    """The series (indices into `shapes`) rank `rank` of `world` reconstructs: the series
    are independent, so they are dealt out with no exchange between ranks -- largest work
    first (voxel-view updates of one iteration) to the rank with the least work so far,
    ties to the lower rank.  Every rank computes the same deal."""
    work = [s[0][0] * s[0][1] * s[0][2] * s[1] for s in shapes]
    load = [0] * world
    owner = [0] * len(shapes)
    for i in sorted(range(len(shapes)), key=lambda i: (-work[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += work[i]
    return [i for i in range(len(shapes)) if owner[i] == rank]


def run_c4(args, rank: int = 0, world: int = 1, local: int = 0):
    """Batched SART of the 64 C4 series (the whole iteration of every series in one
    persistent launch, its launch shape from the autotuner) against the same series one
    after another (one graph per series).  Volumes are FP32 masters with an FP16 shadow
    (the forward projections read FP16 values, updates accumulate in FP32); --c4-f32
    keeps plain FP32 volumes.  Under torchrun each rank batches its share of the 64
    series (c4_shard; strong scaling of the fixed job, no data exchange) and the times are
    the max over ranks."""
    import torch
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BatchReconstructionOperator,
                                          BlockIterativeReconstructionOperator, Context,
                                          ForwardProjectionOperator, GPUMappedVolume, mrc_base_geometry)
    torch.cuda.set_device(local)
    ctx = Context(local)
    dev = torch.device("cuda", local)
    problems = []
    shapes = c4_shapes()
    mine = c4_shard(shapes, rank, world)
    for i in mine:
        (X, Y, Z), nv, tmax = shapes[i]
        ph = make_phantom_torch(4100 + i, dev, (X, Y, Z), count=40, axes=(4.0, 48.0))
        geoms = [mrc_base_geometry(X, Y).rotated(float(a)) for a in np.linspace(-tmax, tmax, nv)]
        vol = GPUMappedVolume(ctx, (X, Y, Z))
        vol.upload(ph.cpu().numpy())
        fp = ForwardProjectionOperator(vol, 1)
        projs = torch.zeros((nv, Y, X), dtype=torch.float32, device=dev)
        scratch = torch.zeros((Y, X), dtype=torch.float32, device=dev)
        for k, g in enumerate(geoms):
            fp.setScannerGeometry(g)
            fp.SetOutput(projs[k], scratch)
            fp.Execute(0)
        vol.close()
        problems.append(((X, Y, Z), geoms, projs.cpu().numpy()))
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=1, lam=LAMBDA, order=_abi.ORDER_IDENTITY)
    stream = torch.cuda.ExternalStream(ctx.stream_handle)
    voxel_type = _abi.VOXEL_FLOAT32 if args.c4_f32 else _abi.VOXEL_F16_MASTER

    def timed(run, reps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.synchronize()
        ev0.record(stream)
        for _ in range(reps):
            run()
        ev1.record(stream)
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / reps

    vols = [GPUMappedVolume(ctx, shape, voxel_type=voxel_type) for shape, _, _ in problems]
    ctx.set_autotune(0 if args.no_autotune else 1)
    batch = BatchReconstructionOperator([(v, g, pr) for v, (_, g, pr) in zip(vols, problems)], p)
    tuned = ctx.tune_report()
    for _ in range(args.warmup):
        batch.runNiterations(1)
    barrier(world)
    with ClockSampler(local) as clk:
        batch_ms = timed(lambda: batch.runNiterations(1), args.steps)
    batch_ms = max_over_ranks(batch_ms, world)
    launches = batch.launches_per_iteration
    batch.close()
    for v in vols:
        v.close()
    seq = []
    ctx.set_autotune(0)
    for shape, geoms, projs in problems:
        vol = GPUMappedVolume(ctx, shape, voxel_type=voxel_type)
        rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
        seq.append((vol, rec))
    def run_seq():
        for _, rec in seq:
            rec.runNiterations(1)
    for _ in range(args.warmup):
        run_seq()
    barrier(world)
    seq_ms = max_over_ranks(timed(run_seq, args.steps), world)
    seq_launches = sum(r.launches_per_iteration for _, r in seq)
    for vol, rec in seq:
        rec.close()
        vol.close()
    # work of the whole job (every rank's series)
    updates = sum(s[0][0] * s[0][1] * s[0][2] * s[1] for s in shapes)
    byts = sum(s[1] * (3 * s[0][0] * s[0][1] * s[0][2] * 4 + 20 * s[0][0] * s[0][1]) for s in shapes)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0)) * world  # the job's bytes over every rank's HBM
    if rank != 0:
        ctx.close()
        return
    print(json.dumps({
        "metric": "C4 batched SART ms per iteration (64 series)", "value": batch_ms, "unit": "ms",
        "higher_is_better": False, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "scaling": "strong", "series_of_rank0": len(mine),
        "dtype": "f32" if args.c4_f32 else "f32 math, f16 shadow, f32 master",
        "tuned_launch_shape": tuned.strip().splitlines(),
        "data": "synthetic (seeded 40-ellipsoid phantoms per series, CUDA-forward-projected, noise-free)",
        "config": {"workload": "C4: 64 SART series, 96^3 to 256x256x128, 41 to 81 views over +-50..70 deg",
                   "series": C4_SERIES, "voxel_view_updates_per_iteration": updates},
        "sequential_ms": seq_ms, "speedup_vs_sequential": seq_ms / batch_ms,
        "launches_per_iteration": {"batched": launches, "sequential": seq_launches},
        "voxel_updates_per_s": updates / (batch_ms * 1e-3),
        "roofline": {"bound": "hbm", "achieved": byts / (batch_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": byts / (batch_ms * 1e-3) / 1e9 / hbm,
                     "bytes": "per view: 4V forward read + 8V back read+write + 20P", "gpus": world},
        "clocks": clk.summary()}))
    ctx.close()


# ------------------------------------------------------------------ C3: perspective, BF16 shadow, block 8
C3_RES = (2048, 2048, 512)
C3_VIEWS = 121


def c3_geometry(tilt: float, res=C3_RES):
    """Perspective view of a res[0] x res[1] detector (2048^2 for C3): source 10 x volume
    width above the volume centre, detector plane one unit from the source with a pitch
    that spans the volume at its centre (the reference's perspective convention,
    ProjectionTestBase.cpp:137-145), rotated by -tilt about y."""
    from ettention_b200.operators import ScannerGeometry
    D = 10.0 * res[0]
    pitch = 1.0 / D
    W, H = res[0], res[1]
    base = ScannerGeometry([0.0, 0.0, D], [-0.5 * W * pitch, -0.5 * H * pitch, D - 1.0], [pitch, 0.0, 0.0],
                           [0.0, pitch, 0.0], W, H, True)
    return base.rotated(tilt)


def run_c3(args, steps=None, warmup=None, cpu_baseline=True):
    """C3: 2048^2 x 512 volume, 121 perspective views (-60..60 step 1), block size 8,
    FP32 master + BF16 shadow, random order, Poisson I0 = 200; one block-iterative
    iteration per step.  Returns the record (clocks, roofline, CPU sample)."""
    import torch
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator, Context,
                                          ForwardProjectionOperator, GPUMappedVolume)
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    ctx = Context(0)
    dev = torch.device("cuda", 0)
    res = tuple(int(v) for v in args.c3_res.split(","))
    X, Y, Z = res
    phantom = make_phantom_torch(3000, dev, res, count=500, axes=(8.0 * X / 2048, 256.0 * X / 2048))
    geoms = [c3_geometry(float(a), res) for a in np.linspace(-60.0, 60.0, C3_VIEWS)]
    vol = GPUMappedVolume(ctx, res)
    host_phantom = phantom.cpu().numpy()
    vol.upload(host_phantom)
    del phantom
    fp = ForwardProjectionOperator(vol, 1)
    projs = torch.zeros((C3_VIEWS, Y, X), dtype=torch.float32, device=dev)
    scratch = torch.zeros((Y, X), dtype=torch.float32, device=dev)
    for i, g in enumerate(geoms):
        fp.setScannerGeometry(g)
        fp.SetOutput(projs[i], scratch)
        fp.Execute(0)
    vol.close()
    gen = torch.Generator(device=dev)
    gen.manual_seed(3000)
    counts = torch.poisson(200.0 * torch.exp(-projs), generator=gen)
    b = (-torch.log(torch.clamp(counts, min=1.0) / 200.0)).contiguous()
    del counts, projs, scratch
    torch.cuda.synchronize()
    cpu_views = None
    if cpu_baseline:
        # three views across the tilt range (-60, 0 and +60 deg): the walk lengths differ
        cpu_views = [(geoms[i], b[i].cpu().numpy()) for i in (0, C3_VIEWS // 2, C3_VIEWS - 1)]
    p = AlgebraicParameterSet(algorithm="blockIterative", block_size=8, iterations=1, lam=0.2,
                              order=_abi.ORDER_RANDOM)
    vol = GPUMappedVolume(ctx, res, voxel_type=_abi.VOXEL_BF16_MASTER)
    rec = BlockIterativeReconstructionOperator(vol, geoms, b, p)
    stream = torch.cuda.ExternalStream(ctx.stream_handle)
    for _ in range(warmup):
        rec.runNiterations(1)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    with ClockSampler(0) as clk:
        ev0.record(stream)
        rec.runNiterations(steps)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    fp_ms, bp_ms, nf, nb = rec.profile_iteration()
    rec.close()
    vol.close()
    ctx.close()
    del b
    V, P, N, B = X * Y * Z, X * Y, C3_VIEWS, 8
    nblocks = (N + B - 1) // B
    # byte model: FP reads the BF16 shadow, b, writes (r, L); BP read-modify-writes the
    # FP32 master once per block and rewrites the shadow; it reads (r, L) per view
    fp_bytes = N * (V * 2 + P * 4 + P * 8)
    bp_bytes = nblocks * (2 * V * 4 + V * 2) + N * P * 8
    byts = fp_bytes + bp_bytes
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    cpu = None
    if cpu_views is not None:
        threads = os.cpu_count() or 1
        t = sum(c3_cpu_seconds_per_view(host_phantom, res, v, threads) for v in cpu_views) / len(cpu_views)
        cpu = {"value": t * N, "unit": "s", "cores": threads, "kind": "port",
               "sample": "3 of the 121 views (-60, 0 and +60 deg: perspective FP + residual + Q8 perspective BP) "
                         "at full size from a zero volume, FP32 oracle; mean seconds per view x121 views"}
    del host_phantom
    return {
        "metric": "C3 block-iterative s per iteration", "value": ms / 1e3, "unit": "s", "higher_is_better": False,
        "n_gpus": 1, "steps": steps, "warmup": warmup, "dtype": "f32 math, bf16 shadow, f32 master",
        "data": "synthetic (seeded 500-ellipsoid phantom, CUDA-forward-projected, Poisson I0=200)",
        "config": {"workload": f"C3: {X}x{Y}x{Z}, 121 perspective views -60..60 step 1, {X}x{Y} detector, "
                               "block 8, lambda 0.2, random order", "voxel_type": "bf16_master",
                   "l2": f"inputs larger than L2 ({V * 6 / 2**30:.1f} GiB volume)"},
        "per_kernel_ms": {"forward_project_total": fp_ms, "back_project_total": bp_ms,
                          "forward_launches": nf, "back_launches": nb},
        "roofline": {"bound": "hbm", "bytes_per_iteration": byts, "achieved": byts / (ms * 1e-3) / 1e9,
                     "peak": hbm, "unit": "GB/s", "frac": byts / (ms * 1e-3) / 1e9 / hbm,
                     "per_kernel": {
                         "forward_project": {"kernel": "forward_project_kernel (perspective walk)",
                                             "algorithmic_bytes": fp_bytes,
                                             "frac": fp_bytes / (fp_ms * 1e-3) / 1e9 / hbm},
                         "back_project": {"kernel": "bp_perspective_kernel", "algorithmic_bytes": bp_bytes,
                                          "frac": bp_bytes / (bp_ms * 1e-3) / 1e9 / hbm}}},
        "cpu_baseline": cpu, "clocks": clk.summary()}


def c3_cpu_seconds_per_view(phantom, res, view, threads: int):
    """Seconds for one C3 view of the FP32 CPU restatement of the reference kernels
    (oracle/) on `threads` host threads: perspective forward projection of a zero volume,
    residual, perspective back projection (texture weights rounded to 1/256)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    g, b = view
    og = O.ScannerGeometry(np.asarray(g.source, np.float64), np.asarray(g.detector, np.float64),
                           np.asarray(g.hpitch, np.float64), np.asarray(g.vpitch, np.float64), g.width, g.height, True)
    vg = O.VolumeGeometry.centered(res)
    vol = np.zeros_like(phantom)
    t0 = time.perf_counter()
    p, l = O.forward_project(vol, vg, og, 1, 32)
    r = b - p
    O.back_project(vol, vg, og, r, l, 0.2 / 8, 1, 32, O.WEIGHTS_Q8)
    return time.perf_counter() - t0


# ------------------------------------------------------------------ C5: learned warm start vs plain SART
def warmstart_flops(res):
    """Multiply-adds x 2 of one inference of the warm-start network (3x3x3 convolutions)."""
    from ettention_b200.learned import LAYERS
    X, Y, Z = res
    level_vox = {1: X * Y * Z, 2: X * Y * Z // 8, 3: X * Y * Z // 64}
    levels = [1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 1]
    return sum(2 * 27 * (c0 + c1) * co * level_vox[l] for (c0, c1, co), l in zip(LAYERS, levels))


def run_c5(args):
    """Held-out series of the learned warm start's workload (256^3/2 volumes, 61 views,
    Poisson 100, SART lambda 0.03): the time plain SART takes to first reach its own
    30-iteration residual ||Ax - b||^2, against 3 plain iterations + the network + the
    residual judge + the plain iterations that then reach the same residual; both timed
    with CUDA events on the library stream (the per-iteration residual checks that find
    the iteration counts run untimed, before the timed runs)."""
    import torch
    from ettention_b200 import warmstart as W
    from ettention_b200.learned import DEFAULT_WEIGHTS, WarmStartNet, load_weights
    from ettention_b200.operators import Context
    if not os.path.exists(DEFAULT_WEIGHTS):
        return {"metric": "C5 learned warm start", "unavailable": "no trained weights file"}
    params, scale, meta = load_weights(DEFAULT_WEIGHTS)
    ctx = Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream_handle)
    net = WarmStartNet(ctx, W.RES, params=params, scale=scale)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    per = []
    cap = 3 * W.TARGET_ITERS
    with ClockSampler(0) as clk:
        for j in range(args.c5_seeds):
            s = W.make_series(ctx, W.HELDOUT_SEED0 + j)
            plain = W.PlainSart(ctx, s)
            plain.set_volume(None)
            r = []
            for _ in range(W.TARGET_ITERS):
                plain.iterate(1)
                r.append(plain.residual())
            target = r[-1]
            k_plain = next(i + 1 for i, x in enumerate(r) if x <= target)
            for _ in range(args.warmup if j == 0 else 0):
                plain.set_volume(None)
                plain.iterate(k_plain)
            plain.set_volume(None)
            t_plain = timed(lambda: plain.iterate(k_plain))
            plain.close()
            solver = W.WarmStartSolver(ctx, net, s)
            kept = solver.start()
            k_ws = 0
            r_ws = solver.residual()
            while r_ws > target and k_ws < cap:
                solver.iterate(1)
                k_ws += 1
                r_ws = solver.residual()
            reached = r_ws <= target
            t_ws = timed(lambda: (solver.start(), solver.iterate(k_ws)))
            t_net = timed(lambda: net.infer(solver.v_in, solver.v_ws, 1))
            per.append({"seed": s.seed, "plain_iters": k_plain, "plain_ms": t_plain, "kept": bool(kept),
                        "judge": [float(x) for x in solver.judge], "extra_iters": k_ws, "reached": bool(reached),
                        "warm_ms": t_ws, "net_ms": t_net, "speedup": t_plain / t_ws,
                        "r3": r[W.INPUT_ITERS - 1], "r30": target})
            solver.close()
            del s
    net.close()
    ctx.close()
    sp = np.array([p["speedup"] for p in per])
    flops = warmstart_flops(W.RES)
    net_ms = float(np.median([p["net_ms"] for p in per]))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    tf_peak = float(peaks.get("bf16_tflops", 1590.0))
    return {
        "metric": "C5 SART s to reach plain 30-iter residual, learned vs plain",
        "value": float(np.median([p["warm_ms"] for p in per])) / 1e3, "unit": "s", "higher_is_better": False,
        "plain_s": float(np.median([p["plain_ms"] for p in per])) / 1e3,
        "speedup_median": float(np.median(sp)), "speedup_mean": float(np.mean(sp)),
        "speedup_min": float(np.min(sp)), "kept_fraction": float(np.mean([p["kept"] for p in per])),
        "reached_fraction": float(np.mean([p["reached"] for p in per])),
        "extra_iters_median": float(np.median([p["extra_iters"] for p in per])),
        "plain_iters_median": float(np.median([p["plain_iters"] for p in per])),
        "n_seeds": len(per), "warmup": args.warmup,
        "config": {"workload": "C5: 256x256x128 ellipsoid phantoms (40, semi-axes 8-64, density 0.05-1 x 0.02), "
                               "61 parallel views -60..60, Poisson I0=100, SART lambda 0.03, identity order; "
                               f"held-out seeds {W.HELDOUT_SEED0}..{W.HELDOUT_SEED0 + len(per) - 1}",
                   "network": "3-level 3-D conv encoder-decoder 16/32/64, BF16, FP32 accumulate",
                   "trained": {k: (v.tolist() if hasattr(v, "tolist") else v) for k, v in meta.items()
                               if k in ("series", "epochs", "lr", "train_seed0")}},
        "roofline": {"bound": "tensor", "kernel": "conv_tc_kernel (network inference)", "flops_per_inference": flops,
                     "achieved": flops / (net_ms * 1e-3) / 1e12, "peak": tf_peak, "unit": "TFLOP/s",
                     "frac": flops / (net_ms * 1e-3) / 1e12 / tf_peak, "net_ms": net_ms},
        "clocks": clk.summary(), "per_seed": per[:8]}


# ------------------------------------------------------------------ blob basis functions
BLOB_RES = (256, 256, 256)
BLOB_VIEWS = 61


def blob_geometry(tilt: float):
    """Perspective view of a 256^2 detector, the source 10 x volume width from the volume
    centre, one detector pixel per voxel at the centre (as c3_geometry), rotated by -tilt."""
    from ettention_b200.operators import ScannerGeometry
    D = 10.0 * BLOB_RES[0]
    pitch = 1.0 / D
    W, H = BLOB_RES[0], BLOB_RES[1]
    base = ScannerGeometry([0.0, 0.0, D], [-0.5 * W * pitch, -0.5 * H * pitch, D - 1.0], [pitch, 0.0, 0.0],
                           [0.0, pitch, 0.0], W, H, True)
    return base.rotated(tilt)


def run_blobs(args):
    """Blob basis functions (algorithm.basisFunctions = blobs): 256^3 Kaiser-Bessel
    coefficients (a = 2, m = 2, alpha = 3.6), 61 perspective views -60..60 step 2, 256^2
    detector, SART (lambda 0.3, random order); one iteration per step."""
    import torch
    from ettention_b200 import _abi
    from ettention_b200.operators import (AlgebraicParameterSet, BlobParameters, BlockIterativeReconstructionOperator,
                                          Context, GPUMappedVolume, forward_project_blobs)
    ctx = Context(0)
    dev = torch.device("cuda", 0)
    X, Y, Z = BLOB_RES
    phantom = make_phantom_torch(5000, dev, BLOB_RES, count=40, axes=(4.0, 64.0))
    geoms = [blob_geometry(float(a)) for a in np.linspace(-60.0, 60.0, BLOB_VIEWS)]
    vol = GPUMappedVolume(ctx, BLOB_RES)
    vol.upload(phantom.cpu().numpy())
    del phantom
    projs = torch.zeros((BLOB_VIEWS, Y, X), dtype=torch.float32, device=dev)
    scratch = torch.zeros((Y, X), dtype=torch.float32, device=dev)
    for i, g in enumerate(geoms):
        forward_project_blobs(vol, g, BlobParameters(), projs[i], scratch)
    vol.close()
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=1, lam=0.3, order=_abi.ORDER_RANDOM,
                              basis_functions="blobs")
    vol = GPUMappedVolume(ctx, BLOB_RES)
    rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
    stream = torch.cuda.ExternalStream(ctx.stream_handle)
    for _ in range(args.warmup):
        rec.runNiterations(1)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    with ClockSampler(0) as clk:
        ev0.record(stream)
        rec.runNiterations(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    fp_ms, bp_ms, nf, nb = rec.profile_iteration()
    rsq = rec.last_residual_sq()
    rec.close()
    vol.close()
    ctx.close()
    # the forward kernel's work: per pixel, every slice along the dominant axis (256 here
    # for every view up to 60 degrees) tests the (2 ceil(1.415 a) + 1)^2 = 49 coefficients
    # around the pierced voxel
    grid = int(np.ceil(np.float32(1.415) * np.float32(2.0)))
    fp_evals = X * Y * Z * (2 * grid + 1) ** 2
    print(json.dumps({
        "metric": "blob SART s per iteration", "value": ms / 1e3, "unit": "s", "higher_is_better": False,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "dtype": "f32",
        "data": "synthetic (seeded 40-ellipsoid phantom as blob coefficients, blob-forward-projected)",
        "config": {"workload": "blobs: 256^3 Kaiser-Bessel coefficients (a=2, m=2, alpha=3.6), 61 perspective "
                               "views -60..60 step 2, 256^2 detector, SART lambda 0.3, random order",
                   "l2": "volume 64 MiB is L2-resident"},
        "per_kernel_ms": {"forward_total": fp_ms, "back_total": bp_ms, "forward_launches": nf, "back_launches": nb,
                          "forward_avg": fp_ms / max(nf, 1), "back_avg": bp_ms / max(nb, 1)},
        "roofline": {"bound": "issue", "forward_coefficient_tests_per_launch": fp_evals,
                     "forward_gtests_per_s": fp_evals / (fp_ms / max(nf, 1) * 1e-3) / 1e9},
        "residual_sq_last_iteration": rsq, "clocks": clk.summary()}))


def run_warmstart_case():
    """Three inferences of the trained warm-start network on one held-out 3-iteration SART
    volume (the case the convolution kernels are profiled on)."""
    import torch
    from ettention_b200 import warmstart as W
    from ettention_b200.learned import WarmStartNet, load_weights
    from ettention_b200.operators import Context
    params, scale, _ = load_weights()
    ctx = Context(0)
    s = W.make_series(ctx, W.HELDOUT_SEED0)
    v3, = W.sart_pair(ctx, s, stops=(W.INPUT_ITERS,))
    net = WarmStartNet(ctx, W.RES, params=params, scale=scale)
    x = v3[None].contiguous()
    y = torch.empty_like(x)
    stream = torch.cuda.ExternalStream(ctx.stream_handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(3):
        if i == 2:
            e0.record(stream)
        net.infer(x, y)
    e1.record(stream)
    e1.synchronize()
    net.check()
    print(json.dumps({"warmstart_case": "256x256x128, one held-out 3-iteration SART volume",
                      "infer_ms": e0.elapsed_time(e1), "flops": warmstart_flops(W.RES)}))
    net.close()
    ctx.close()


def main():
    args = parse()
    if args.warmstart_case:
        run_warmstart_case()
        return
    if args.ncu_case:
        run_ncu_case(tuple(int(v) for v in args.ncu_res.split(",")))
        return

    if args.workload == "c3":
        print(json.dumps(run_c3(args, cpu_baseline=not args.no_cpu_baseline)), flush=True)
        return
    if args.workload == "c5":
        print(json.dumps(run_c5(args)), flush=True)
        return
    if args.workload == "blobs":
        run_blobs(args)
        return
    rank, world, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "slabs":
            run_slabs(args, rank, world, local)
        elif args.workload == "c4":
            run_c4(args, rank, world, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
