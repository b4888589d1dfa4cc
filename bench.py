#!/usr/bin/env python
"""Benchmark of the multi-view reconstruction path on B200.

Workload (the transform + plain-RL configuration): 4 raw views, uint16
512 x 512 x 128 with z spacing 3 (seeded synthetic beads and shells, blurred
per plane, Poisson noise); inverse affines = rotation about y by
0/90/180/270 degrees, z scale 3, shift U[-8, 8]; trilinear resampling of each
view into a 512 x 512 x 384 common frame (uint16, as the reference API
produces); weights = the transformed masks (border 16); then 20 plane-wise
RL iterations with 31 x 31 anisotropic Gaussian kernels (sigma 1.2 x 5.0,
rotated per view), FP32.  A step is one such volume: resample all views and
deconvolve all 384 planes.

Metric: RL voxel-iter/s = 512 * 512 * 384 frame voxels * 20 iterations /
step time.  'value' is measured with inputs resident in device memory (CUDA
events on the launch stream); 'e2e' through the C ABI with host buffers
(transform_host, then fmvd_initialize / deconvolve_planes / destroy with a
datasource and datasink on host memory).  Inputs (268 MB of source views)
exceed the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one rank per GPU) every rank deconvolves its own
volume (weak scaling); the time is the maximum over ranks.  --impl reference
times the reference's own implementation of the path: the reference CUDA
library built from the upstream sources (cuFFT) for the deconvolution and the
texture-unit restatement of its resampler, through their host-memory API.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

V = 4
SRC = (128, 512, 512)     # d, h, w of each raw view
FRAME = (384, 512, 512)   # td, th, tw
ITERATIONS = 20
KSIZE = 31
ZSCALE = 3.0
BORDER = 16
BYTES_PER_PADDED_VOXEL_VIEW_ITER = 14  # read e (4) + write e (4) + data (2) + weight (4)
METRIC = "RL voxel-iter/s"
WORKLOAD_NAME = ("transform + plain RL: 4 views u16 512x512x128 (z spacing 3) -> 512x512x384 frame, 20 RL "
                 "iterations, 31x31 PSFs, FFT plane 1024x1024")
UNIT = "voxel-iter/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--small", action="store_true", help="small volume for profiler captures")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--workload", default="transform_rl", choices=["transform_rl", "warmstart", "batched", "planes", "large"],
                   help="warmstart: learned warm start vs plain RL-50 (time to the RL-50 result); planes: plain "
                        "RL throughput per padded plane size (--planes); large: the large streamed configuration "
                        "(run with --steps 1 --warmup 1: one step takes tens of seconds)")
    p.add_argument("--planes", default="1400,2048",
                   help="planes workload: comma-separated data plane sizes, each padded by a 31 x 31 kernel "
                        "(63 x 63 from 2000 up): 900 -> 1024, 1400 -> 1536, 2048 -> 2560 FFT planes")
    p.add_argument("--pairs-per-batch", type=int, default=0,
                   help="planes workload: plane pairs per batch (0: the library's default)")
    p.add_argument("--no-warmstart", action="store_true", help="skip the learned warm-start comparison")
    p.add_argument("--large-train-planes", type=int, default=384,
                   help="large workload: frame planes whose 512 x 512 crops train the warm-start network")
    p.add_argument("--large-epochs", type=int, default=12)
    p.add_argument("--large-target-iterations", type=int, default=40,
                   help="large workload: RL iterations of the warm-start training targets")
    p.add_argument("--train-planes", type=int, default=4000)
    # 16 epochs on RL-48 targets: over 2 seeds x 3 targets (42, 46, 48), 16
    # epochs kept every network within 0.9 % of RL-50 on the tuning planes at
    # its best k, 12 epochs only half of them
    p.add_argument("--epochs", type=int, default=16)
    p.add_argument("--target-iterations", type=int, default=48,
                   help="warm start: RL iterations of the training targets (the network then needs 50 - this)")
    return p.parse_args()


# ------------------------------------------------------------------ data
def workload(seed: int, small: bool):
    """Seeded synthetic views, matrices and kernels (numpy + torch on the GPU
    for the blur; data generation only)."""
    import torch
    from gpu_deconvolution_b200 import synth
    src = (SRC[0] // 8, SRC[1], SRC[2]) if small else SRC
    frame = (FRAME[0] // 8, FRAME[1], FRAME[2]) if small else FRAME
    rng = np.random.default_rng(seed)
    gt = synth.bead_volume(src, 2000 if not small else 250, rng, shells=3)
    psfs = [synth.gaussian_psf(KSIZE, KSIZE, 1.2, 5.0, 180.0 * v / V) for v in range(V)]
    g = torch.Generator(device="cuda").manual_seed(seed)
    vols = []
    gtt = torch.from_numpy(gt).cuda()
    d, h, w = src
    for v in range(V):
        k = torch.from_numpy(psfs[v]).cuda()
        fh, fw = h + KSIZE - 1, w + KSIZE - 1
        spec = torch.fft.rfft2(k, s=(fh, fw))
        out = torch.empty_like(gtt)
        for z0 in range(0, d, 32):
            blk = torch.fft.irfft2(torch.fft.rfft2(gtt[z0:z0 + 32], s=(fh, fw)) * spec, s=(fh, fw))
            out[z0:z0 + 32] = blk[:, KSIZE // 2:KSIZE // 2 + h, KSIZE // 2:KSIZE // 2 + w]
        noisy = torch.poisson(out.clamp_min(0), generator=g)
        vols.append(noisy.clamp(0, 65535).round().to(torch.int32).cpu().numpy().astype(np.uint16))
    shifts = rng.uniform(-8, 8, (V, 3))
    mats = [synth.rotation_y_inverse(90.0 * v, frame, src, ZSCALE, shifts[v]) for v in range(V)]
    return vols, mats, psfs, src, frame


def masks_for(mats, src, frame):
    import torch
    from gpu_deconvolution_b200 import api
    out = []
    for m in mats:
        t = torch.zeros((frame[1], frame[2]), dtype=torch.float32, device="cuda")
        api.mask_device(t, frame[0] // 2, src[2], src[1], src[0], ZSCALE, frame[2], frame[1], BORDER, m)
        torch.cuda.synchronize()
        out.append(t.cpu().numpy().astype(np.float32))
    return out


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling during the timed region (200 ms period)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- utilities
def peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the four
# passes of one view update of a 6-plane batch of 1024 x 1024 planes, per
# padded voxel, from one ncu capture of this workload's small case:
#   ncu --set full --cache-control none --clock-control none \
#       -k regex:"row_pass_w|col_pass_w" -s 40 -c 4 \
#       python bench.py --small --steps 1 --warmup 1 --no-e2e --no-cpu
# (22.1 MB per view update; the batch's work planes stay in L2).
DRAM_BYTES_PER_PADDED_VOXEL_VIEW_UPDATE = 3.52
# Thread instructions of the same four passes per padded voxel (the same
# capture's smsp__inst_executed.sum x 32 / padded voxels: 38.62 M warp
# instructions per view update of the 6-plane batch).  With one warp
# instruction per SM sub-partition per cycle (148 SMs x 4 x 32 lanes x clock)
# this gives the issue-bound ceiling of the passes.
THREAD_INSTR_PER_PADDED_VOXEL_VIEW_UPDATE = 196.3


def dist_setup(n):
    import torch
    if n <= 1 or "WORLD_SIZE" not in os.environ:
        return 0, 1, 0
    import datetime
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    return rank, world, local


def barrier_max(t, world):
    import torch
    if world <= 1:
        return t
    import torch.distributed as dist
    x = torch.tensor([t], dtype=torch.float64, device="cuda")
    dist.all_reduce(x, op=dist.ReduceOp.MAX)
    return float(x.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------- CPU baseline
def cpu_baseline(vols, weights, psfs, iterations=4, label=None):
    """The C/OpenMP port of the per-plane update (oracle/fmvd_cpu.c) on a
    bounded sample: one plane pair per host thread (at most 96 planes),
    ``iterations`` iterations, all views, on the workload's plane geometry.
    vols: per-view frame planes (D x H x W uint16 arrays)."""
    import ctypes as C
    from oracle import fmvd_oracle as O
    path = os.path.join(ROOT, "oracle", "_build", "libfmvd_cpu.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    threads = int(lib.fmvdcpu_max_threads())
    planes = min(2 * threads, 96)
    nv = len(psfs)
    H, W = vols[0].shape[1:]
    kH, kW = psfs[0].shape
    sample = np.ascontiguousarray(np.stack([v[:planes] if v.shape[0] >= planes else np.resize(v, (planes, H, W))
                                            for v in vols]))
    k1 = np.stack([O.normalize(p) for p in psfs]).astype(np.float32)
    k2 = np.stack(O.compute_kernel2(psfs, 0)).astype(np.float32)
    w = np.ascontiguousarray(np.stack(weights).astype(np.float32))
    out = np.zeros((planes, H, W), np.uint16)
    P = lambda a: C.c_void_p(a.ctypes.data)
    t0 = time.perf_counter()
    lib.fmvdcpu_deconvolve(16, P(sample), P(w), P(k1), P(k2), nv, planes, H, W, kH, kW, iterations, P(out), None,
                           threads)
    dt = time.perf_counter() - t0
    fh, fw = O.snap_transform_size(H + kH - 1), O.snap_transform_size(W + kW - 1)
    return {"value": H * W * planes * iterations / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"C/OpenMP port of the per-plane update, {planes} planes x {iterations} iterations x {nv} views "
                      f"at {H}x{W} ({fh}x{fw} padded), {dt:.1f} s"}


# ---------------------------------------------------------------- B200
def run_b200(args):
    import torch
    from gpu_deconvolution_b200 import api, native
    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    lib = native.load()
    vols, mats, psfs, src, frame = workload(1234 + rank, args.small)
    weights = masks_for(mats, src, frame)
    d, h, w = src
    td, th, tw = frame
    pitch = api.source_pitch(16, w)
    src_dev = torch.zeros((V, d, h, pitch), dtype=torch.int16, device="cuda")
    for v in range(V):
        src_dev[v, :, :, :w] = torch.from_numpy(vols[v].view(np.int16)).cuda()
    frame_dev = torch.zeros((V, td, th, tw), dtype=torch.int16, device="cuda")
    out_dev = torch.zeros((td, th, tw), dtype=torch.int16, device="cuda")
    plan = api.DevicePlan(th, tw, weights, [p.copy() for p in psfs], 0, bits=16)
    stream = torch.cuda.current_stream().cuda_stream

    def step(ev=None):
        for v in range(V):
            api.transform_device(src_dev[v], pitch, w, h, d, mats[v], tw, th, 0, td, out=frame_dev[v], stream=stream)
        if ev:
            ev[0].record()
        plan.run(frame_dev, out_dev, ITERATIONS, stream=stream)
        if ev:
            ev[1].record()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = lib.fmvd_b200_launch_count()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    rl_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                 for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        e_start.record()
        for i in range(args.steps):
            step(rl_events[i])
        e_end.record()
        torch.cuda.synchronize()
    launches = lib.fmvd_b200_launch_count() - launches0
    t_total = e_start.elapsed_time(e_end) / 1e3
    t_rl = sum(a.elapsed_time(b) for a, b in rl_events) / 1e3
    barrier(world)
    t_max = barrier_max(t_total, world)
    voxel_iters = td * th * tw * ITERATIONS
    value = voxel_iters * args.steps * world / t_max

    # roofline of the fused RL passes (algorithmic bytes per padded voxel, view and iteration)
    H, W = plan.fftH, plan.fftW
    alg_bytes = BYTES_PER_PADDED_VOXEL_VIEW_ITER * H * W * td * V * ITERATIONS * args.steps
    achieved = alg_bytes / t_rl / 1e9
    peak, peak_kind = peak_hbm()
    # one unit of the roofline = one view update of one batch of plane pairs
    # (the four passes row divide, column K^, row update, column K)
    batch_planes = 2 * plan.pairs_per_batch
    n_updates = -(-td // batch_planes) * V * ITERATIONS * args.steps
    alg_per_update = BYTES_PER_PADDED_VOXEL_VIEW_ITER * H * W * batch_planes
    traffic_per_update = DRAM_BYTES_PER_PADDED_VOXEL_VIEW_UPDATE * H * W * batch_planes

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, vols, mats, psfs, weights, src, frame, world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        frames = frame_dev[:, :min(96, td)].cpu().numpy().view(np.uint16)
        cpu = cpu_baseline(list(frames), weights, psfs)
    warm = None
    if rank == 0 and world == 1 and not args.no_warmstart and not args.small:
        # the metric's second half: time to the plain RL-50 result, learned
        # warm start vs plain RL (its own workload, after the timed region)
        del frame_dev, src_dev, out_dev
        torch.cuda.empty_cache()
        try:
            warm = warmstart_result(args, log=False)
        except Exception as exc:  # reported in the line, never hides the RL figures
            warm = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME + (" [small]" if args.small else ""),
                       "views": V, "frame": list(frame), "iterations": ITERATIONS, "fft_plane": [H, W],
                       "pairs_per_batch": plan.pairs_per_batch,
                       "l2": "inputs larger than L2 (268 MB of source views per step)",
                       "rl_ms_per_step": t_rl / args.steps * 1e3,
                       "transform_ms_per_step": (t_total - t_rl) / args.steps * 1e3},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "kernel": "fused RL view update (row divide, column K^, row update, column K passes)",
                         "unit_of_work": f"one view update of a batch of {batch_planes} padded planes",
                         "algorithmic_bytes_per_update": alg_per_update,
                         "update_ms": t_rl / n_updates * 1e3,
                         "algorithmic_bytes": "14 B per padded voxel per view per iteration",
                         "traffic": traffic_per_update,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the four passes of "
                                           "one view update, small case of this workload (same batch shape)"},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "warmstart": warm,
        }
        clk_sum = line["clocks"]
        mhz = clk_sum.get("sm_mhz") or 1965.0
        issue_rate = 148 * 4 * 32 * mhz * 1e6            # thread instructions per second
        ceiling = issue_rate / THREAD_INSTR_PER_PADDED_VOXEL_VIEW_UPDATE   # padded voxel-view-updates/s
        rate = alg_bytes / BYTES_PER_PADDED_VOXEL_VIEW_ITER / t_rl
        line["roofline"]["issue_ceiling"] = {
            "padded_voxel_view_updates_per_s": ceiling, "achieved": rate, "frac": rate / ceiling,
            "as_hbm_frac": ceiling * BYTES_PER_PADDED_VOXEL_VIEW_ITER / 1e9 / peak,
            "model": f"{THREAD_INSTR_PER_PADDED_VOXEL_VIEW_UPDATE} thread instructions per padded voxel per view "
                     f"update (ncu) at one warp instruction per SM sub-partition per cycle, {mhz:.0f} MHz"}
        print(json.dumps(line), flush=True)
    plan.destroy()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_e2e(args, vols, mats, psfs, weights, src, frame, world=1):
    """The same step end to end through the C ABI with host buffers: pinned
    source volumes in, the result in host memory out
    (fmvd_b200_reconstruct_host: sources uploaded once, resampling and RL in
    chunks on the device, result chunks copied back while the next chunk
    computes).  The reference-compatible path (transform_cuda-style output to
    the host, then the streaming datasource/datasink API) is timed beside it
    for one step."""
    import torch
    from gpu_deconvolution_b200 import api
    td, th, tw = frame
    pinned = [torch.from_numpy(v.view(np.int16)).pin_memory().numpy().view(np.uint16) for v in vols]
    out = np.empty(frame, np.uint16)
    plan = api.DevicePlan(th, tw, weights, [p.copy() for p in psfs], 0, bits=16)
    rec = api.Reconstructor(plan, V, src, frame)
    try:
        rec.run(pinned, mats, ITERATIONS, out)
        n = max(1, min(args.steps, 3))
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(n):
            rec.run(pinned, mats, ITERATIONS, out)
        dt = barrier_max((time.perf_counter() - t0) / n, world)  # slowest rank
    finally:
        rec.destroy()
        plan.destroy()
    d = src[0]
    h2d = V * d * src[1] * src[2] * 2
    d2h = td * th * tw * 2

    # the drop-in path as a C program drives it (C datasource and datasink):
    # resample every view into host memory, then stream the planes through
    # fmvd_initialize / deconvolve_planes / destroy_cuda_16 with nstreams 3
    frames = np.empty((V, td, th, tw), np.uint16)
    for _ in range(2):  # the first run also pages in the host buffers
        t0 = time.perf_counter()
        for v in range(V):
            api.transform_host(pinned[v], mats[v], tw, th, td, out=frames[v])
        t1 = time.perf_counter()
        ref_api_out = api.deconvolve_c_callbacks(frames, weights, [p.copy() for p in psfs], 0, ITERATIONS,
                                                 nstreams=3)
        t2 = time.perf_counter()
        assert ref_api_out.shape[0] == td
    dt_ref_api = t2 - t0
    return {"value": td * th * tw * ITERATIONS * world / dt, "unit": UNIT, "h2d_bytes_per_step": h2d * world,
            "d2h_bytes_per_step": d2h * world, "ms_per_step": dt * 1e3,
            "api": "fmvd_b200_reconstruct_host (pinned sources in, result to host memory)",
            "reference_style_api": {
                "value": td * th * tw * ITERATIONS / dt_ref_api, "ms_per_step": dt_ref_api * 1e3, "gpus": 1,
                "transform_ms": (t1 - t0) * 1e3, "deconvolve_ms": (t2 - t1) * 1e3,
                "api": "fmvd_b200_transform_host x4 + fmvd_initialize/deconvolve_planes/destroy_cuda_16 "
                       "(frame through host memory, C datasource and datasink, nstreams 3)",
                "h2d_bytes_per_step": h2d + V * td * th * tw * 2, "d2h_bytes_per_step": V * td * th * tw * 2 + d2h}}


# ------------------------------------------------------------ reference
def run_reference(args):
    """The reference's own implementation of the path, timed on the same
    workload: the upstream deconvolution sources built for sm_100a with cuFFT
    (oracle/_ref/libfmvd_ref.so, through fmvd_initialize / deconvolve_planes /
    destroy with C callbacks, nstreams 3) and the texture-unit restatement of
    its resampler and mask kernel (oracle/_ref/libfmvd_reftex.so), host
    buffers in and out.  Nothing of this project's library is loaded."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref_lib as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build (oracle/_ref) not present"}))
        return
    import torch
    torch.cuda.set_device(0)
    lib, tex = R.load_ref()
    vols, mats, psfs, src, frame = workload(1234, args.small)
    d, h, w = src
    td, th, tw = frame
    weights = [R.ref_mask(tex, m, td // 2, w, h, d, ZSCALE, tw, th, BORDER) for m in mats]

    def step():
        frames = np.stack([R.ref_transform(tex, vols[v], mats[v], tw, th, td) for v in range(V)])
        res = R.ref_deconvolve(lib, frames, weights, [p.copy() for p in psfs], 0, ITERATIONS, 3, False)
        assert res["out"].shape[0] == td
        return res["out"]

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step()
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    dt = sum(times) / len(times)
    value = td * th * tw * ITERATIONS / dt
    h2d = V * d * h * w * 2 + V * td * th * tw * 2
    d2h = V * td * th * tw * 2 + td * th * tw * 2
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME + (" [small]" if args.small else ""),
                   "views": V, "frame": list(frame), "iterations": ITERATIONS},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "the whole workload per step through the reference's own implementation, which "
                                   "is CUDA: upstream deconvolution sources built for sm_100a with cuFFT (nstreams 3, "
                                   "C callbacks) and the texture-unit restatement of its resampler and mask, host "
                                   "buffers in and out, one host thread driving 1 B200"},
    }), flush=True)


def unet_flops_per_plane(H, W, V=4, base=32):
    """Multiply-add FLOPs (x 2) of one plane through the network's
    convolutions: forward, and forward + data + weight gradients."""
    shapes = [(64, base, 1), (base, base, 9)]
    for l in range(1, 4):
        shapes += [(base << (l - 1), base << l, 9), (base << l, base << l, 9)]
    for l in (2, 1, 0):
        shapes += [(base << (l + 1), base << l, 9), (base << l, base << l, 9)]
    levels = [0, 0] + [l for l in range(1, 4) for _ in (0, 1)] + [l for l in (2, 1, 0) for _ in (0, 1)]
    fwd = train = 0.0
    for i, ((cin, cout, taps), l) in enumerate(zip(shapes, levels)):
        f = 2.0 * (H >> l) * (W >> l) * cout * taps * cin
        fwd += f
        train += f * (2 if i == 0 else 3)
    return fwd, train


def run_warmstart(args):
    print(json.dumps(warmstart_result(args)), flush=True)


K_TUNE_MARGIN = 0.95  # warm-start k is tuned to this fraction of the tolerance
WARM_SEEDS = 3       # networks trained at most, until one meets the margin


def warmstart_result(args, log=True):
    """Learned warm start (a 2-D U-Net on the tensor cores) vs plain RL-50 on
    512 x 512 planes of 4 views: train on plain RL-N targets (N =
    --target-iterations, a little under 50 so that k RL iterations after the
    network's estimate land on RL-50), tune k so that
    warm start + RL-k is within 0.95e-2 relative L2 of plain RL-50 on its own
    planes, then time both paths to the RL-50 result on test planes, where the
    tolerance is 1e-2."""
    import torch
    from gpu_deconvolution_b200 import api
    from gpu_deconvolution_b200 import warmstart as WS
    H = W = 512
    V, N_RL, TOL = 4, 50, 1e-2
    n_train = args.train_planes
    t0 = time.perf_counter()
    views, targets, gt, psfs = WS.training_pairs(n_train, H, W, V, args.target_iterations, seed=1000,
                                                 planes_per_volume=64)
    t_data = time.perf_counter() - t0
    tv, tt, tg, _ = WS.training_pairs(64, H, W, V, N_RL, seed=900000, planes_per_volume=64)   # k tuning
    ev, et, eg, _ = WS.training_pairs(64, H, W, V, N_RL, seed=950000, planes_per_volume=64)   # test
    plan = api.DevicePlan(H, W, WS.equal_weights(H, W, V), [p.copy() for p in psfs], 0)
    fwd_f, train_f = unet_flops_per_plane(H, W, V)
    # Training (timed on the device, steps of 16 planes), then k tuned on its
    # own planes to 95 % of the tolerance, so that the held-out test planes
    # (a different sample) stay within it.  The atomics of the weight
    # gradients make each training a little different; a network whose
    # tuning planes do not come within the margin at any k is replaced by
    # one trained from the next seed (model selection on the tuning planes
    # only), up to WARM_SEEDS networks.
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_train, trained = 0.0, []
    for seed in range(WARM_SEEDS):
        net = WS.WarmStartNet(H, W, V, max_batch=16, seed=seed)
        e0.record()
        hist = WS.train(net, views, targets, epochs=args.epochs, batch=16, lr=1e-3, seed=seed,
                        log=(lambda m: print(m, file=sys.stderr, flush=True)) if log else None)
        e1.record()
        torch.cuda.synchronize()
        t_train += e0.elapsed_time(e1) / 1e3
        k, k_errors = WS.tune_k(net, plan, tv, tt, K_TUNE_MARGIN * TOL,
                                candidates=tuple(range(0, 13)) + (14, 16, 20, 25, 30, 40))
        trained.append({"seed": seed, "k": k, "best_tuning_rel_l2": min(k_errors.values())})
        if k is not None or seed == WARM_SEEDS - 1:
            break
        net.destroy()
    steps = args.epochs * (n_train // 16) * len(trained)
    del views, targets, gt
    torch.cuda.empty_cache()
    kk = k if k is not None else N_RL
    # time to the RL-50 result on the test planes
    t_plain = WS.time_cuda(lambda: WS.rl_planes(plan, ev, N_RL))
    t_warm = WS.time_cuda(lambda: WS.warm_deconvolve(net, plan, ev, kk))
    t_net = WS.time_cuda(lambda: net.forward(ev))
    warm, _ = WS.warm_deconvolve(net, plan, ev, kk)
    plain, _ = WS.rl_planes(plan, ev, N_RL)
    err = WS.rel_l2_planes(warm.contiguous(), et)
    psnr_plain = WS.psnr(plain, eg)
    psnr_warm = WS.psnr(warm, eg)
    net.check()
    line = {
        "metric": "time to the plain RL-50 result, warm start vs plain", "unit": "ms per 64 planes",
        "value": t_warm, "plain_rl50_ms": t_plain, "speedup": t_plain / t_warm, "k": k,
        "rel_l2_vs_rl50": {"max": float(err.max()), "mean": float(err.mean()), "tolerance": TOL,
                           "k_tuned_to": K_TUNE_MARGIN * TOL},
        "psnr_db": {"plain_rl50": psnr_plain, "warm": psnr_warm, "delta": psnr_warm - psnr_plain},
        "k_search": {str(a): b for a, b in k_errors.items()},
        "network_ms_per_64_planes": t_net,
        "network_tflops": fwd_f * 64 / (t_net / 1e3) / 1e12,
        "training": {"planes": n_train, "target_rl_iterations": args.target_iterations, "epochs": args.epochs,
                     "batch": 16, "steps": steps, "seconds": t_train,
                     "tflops": train_f * 16 * steps / t_train / 1e12, "loss_per_epoch": hist,
                     "data_seconds": t_data, "networks": trained},
        "dtype": "bf16 network (fp32 accumulation), f32 RL", "data": "synthetic",
        "config": {"workload": "learned warm start: 4 views u16 512x512 planes, 17x17 PSFs sigma 1.5x4.0, "
                               f"trained on plain RL-{args.target_iterations} targets, compared with plain RL-50, "
                               "U-Net 4 levels base 32", "fft_plane": [plan.fftH, plan.fftW]},
    }
    plan.destroy()
    net.destroy()
    torch.cuda.empty_cache()
    return line


def run_batched(args):
    """Batched uneven plain RL: 32 independent volumes (planes 128..1024
    square, depths 16..256, 2-6 views, kernels 9..41, 25 iterations) run by
    one CUDA graph launch (fmvd_b200_batch_*), against the same volumes run
    one after another.  (Per-volume errors against the FP64 oracle are
    checked by tests/test_batch_tune.py.)"""
    import torch
    from gpu_deconvolution_b200 import api
    from gpu_deconvolution_b200 import synth as S
    specs = S.batched_specs(0, 32)
    plans, views, outs = [], [], []
    for sp in specs:
        w = [np.ones((sp["H"], sp["W"]), np.float32)] * sp["V"]
        plans.append(api.DevicePlan(sp["H"], sp["W"], w, S.spec_psfs(sp), 0))
        views.append(S.views_torch(sp))
        outs.append(torch.zeros((sp["D"], sp["H"], sp["W"]), dtype=torch.int16, device="cuda"))
    torch.cuda.synchronize()
    its = [sp["iterations"] for sp in specs]
    voxel_iters = sum(sp["D"] * sp["H"] * sp["W"] * sp["iterations"] for sp in specs)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    by_branches = {}
    for nb in (1, 2, 4, 8):
        batch = api.Batch(plans, views, outs, its, max_branches=nb)
        batch.run()
        torch.cuda.synchronize()
        e0.record()
        batch.run()
        e1.record()
        torch.cuda.synchronize()
        by_branches[nb] = e0.elapsed_time(e1)
        batch.destroy()
    best = min(by_branches, key=by_branches.get)
    t_graph = by_branches[best] / 1e3
    # every volume on its own (CUDA events around each run), grouped by
    # padded plane: the graph launch against the sum of the volumes' own
    # times, and each plane class's throughput
    per_class = {}
    t_seq = 0.0
    for sp, p, v, o, it in zip(specs, plans, views, outs, its):
        e0.record()
        p.run(v, o, it)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        t_seq += ms / 1e3
        c = per_class.setdefault(f"{p.fftH}x{p.fftW}", {"volumes": 0, "ms": 0.0, "padded_voxel_view_iters": 0})
        c["volumes"] += 1
        c["ms"] += ms
        c["padded_voxel_view_iters"] += p.fftH * p.fftW * sp["D"] * sp["V"] * it
    for c in per_class.values():
        c["G_padded_voxel_view_iter_per_s"] = c["padded_voxel_view_iters"] / (c["ms"] * 1e-3) / 1e9
    for p in plans:
        p.destroy()
    print(json.dumps({
        "metric": "RL voxel-iter/s, 32 uneven volumes in one graph launch", "unit": UNIT,
        "value": voxel_iters / t_graph, "ms": t_graph * 1e3, "branches": best,
        "ms_by_branches": by_branches, "sequential_ms": t_seq * 1e3,
        "graph_speedup": t_seq / t_graph, "per_plane_class": per_class, "volumes": len(specs),
        "voxel_iters": voxel_iters, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched uneven plain RL (32 volumes, planes 128..1024, depths 16..256, 2-6 views, "
                               "kernels 9..41, 25 iterations)"}}), flush=True)


# Large streamed configuration: 6 views, u16 2048 x 2048 x 512 each, beads and
# shells (1e5 beads), rotations about y 60 degrees apart, z spacing 1.5,
# resampled into a 2048 x 2048 x 768 frame, 63 x 63 PSFs (sigma 2 x 8,
# rotated per view), 50 RL iterations; FFT plane 2560 x 2560.
LARGE_V = 6
LARGE_SRC = (512, 2048, 2048)
LARGE_FRAME = (768, 2048, 2048)
LARGE_K = 63
LARGE_ITERATIONS = 50
LARGE_ZSCALE = 1.5
LARGE_BEADS = 100000
LARGE_NAME = ("large streamed: 6 views u16 2048x2048x512 (z spacing 1.5) in pinned host memory -> 2048x2048x768 "
              "frame, 50 RL iterations, 63x63 PSFs, FFT plane 2560x2560")


def large_workload(seed: int):
    """Seeded synthetic views of the large configuration, generated on the
    GPU and kept in pinned host memory (25.8 GB), plus matrices and PSFs."""
    import torch
    from gpu_deconvolution_b200 import synth
    d, h, w = LARGE_SRC
    gt, g = synth.bead_volume_torch(d, h, w, seed, "cuda", LARGE_BEADS / float(d * h * w))
    synth.add_shells_torch(gt, 3, seed)
    psfs = [synth.gaussian_psf(LARGE_K, LARGE_K, 2.0, 8.0, 180.0 * v / LARGE_V) for v in range(LARGE_V)]
    pinned = []
    for v in range(LARGE_V):
        view = synth.blur_noise_torch(gt, [psfs[v]], g)[0]
        host = torch.empty((d, h, w), dtype=torch.int16, pin_memory=True)
        host.copy_(view)
        pinned.append(host)
        del view
    del gt
    torch.cuda.empty_cache()
    shifts = np.random.default_rng(seed).uniform(-8, 8, (LARGE_V, 3))
    mats = [synth.rotation_y_inverse(360.0 * v / LARGE_V, LARGE_FRAME, LARGE_SRC, LARGE_ZSCALE, shifts[v])
            for v in range(LARGE_V)]
    return pinned, mats, psfs


def run_large(args):
    """The large streamed configuration on one GPU.  'value': sources resident
    on the device, all views resampled into the whole frame and 50 RL
    iterations over its 768 planes (CUDA events).  'e2e': the same through
    fmvd_b200_reconstruct_host with the sources in pinned host memory (upload
    overlapped with the first resampling, result chunks copied back while the
    next chunk computes).  One step takes tens of seconds; inputs (77 GB on
    the device) exceed L2 many times over, so no flush is needed."""
    import torch
    from gpu_deconvolution_b200 import api, native
    lib = native.load()
    V, (d, h, w), (td, th, tw), IT = LARGE_V, LARGE_SRC, LARGE_FRAME, LARGE_ITERATIONS
    t0 = time.perf_counter()
    pinned, mats, psfs = large_workload(4321)
    t_data = time.perf_counter() - t0
    weights = []
    for m in mats:
        t = torch.zeros((th, tw), dtype=torch.float32, device="cuda")
        api.mask_device(t, td // 2, w, h, d, LARGE_ZSCALE, tw, th, BORDER, m)
        weights.append(t.cpu().numpy())
    plan = api.DevicePlan(th, tw, weights, [p.copy() for p in psfs], 0, bits=16)
    pitch = api.source_pitch(16, w)
    stream = torch.cuda.current_stream().cuda_stream
    src_dev = torch.zeros((V, d, h, pitch), dtype=torch.int16, device="cuda")
    for v in range(V):
        src_dev[v, :, :, :w].copy_(pinned[v])
    frame_dev = torch.zeros((V, td, th, tw), dtype=torch.int16, device="cuda")
    out_dev = torch.zeros((td, th, tw), dtype=torch.int16, device="cuda")

    def step(ev):
        ev[0].record()
        for v in range(V):
            api.transform_device(src_dev[v], pitch, w, h, d, mats[v], tw, th, 0, td, out=frame_dev[v], stream=stream)
        ev[1].record()
        plan.run(frame_dev, out_dev, IT, stream=stream)
        ev[2].record()

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.warmup + args.steps)]
    for i in range(args.warmup):
        step(evs[i])
    torch.cuda.synchronize()
    launches0 = lib.fmvd_b200_launch_count()
    with ClockSampler(0) as clk:
        for i in range(args.warmup, args.warmup + args.steps):
            step(evs[i])
        torch.cuda.synchronize()
    launches = lib.fmvd_b200_launch_count() - launches0
    timed = evs[args.warmup:]
    t_total = sum(e[0].elapsed_time(e[2]) for e in timed) / 1e3
    t_rl = sum(e[1].elapsed_time(e[2]) for e in timed) / 1e3
    t_tr = t_total - t_rl
    frames_cpu = [frame_dev[v, :96].cpu().numpy().view(np.uint16) for v in range(V)] if not args.no_cpu else None
    del src_dev
    warm = None
    if not args.no_warmstart:
        try:
            warm = large_warmstart(args, plan, frame_dev)
        except Exception as exc:  # reported in the line, never hides the RL figures
            warm = {"error": f"{type(exc).__name__}: {exc}"}
    del frame_dev, out_dev
    torch.cuda.empty_cache()

    voxel_iters = td * th * tw * IT
    H, W = plan.fftH, plan.fftW
    alg = BYTES_PER_PADDED_VOXEL_VIEW_ITER * H * W * td * V * IT * args.steps
    peak, peak_kind = peak_hbm()
    tr_bytes = V * (d * h * w * 2 + td * th * tw * 2) * args.steps

    e2e = None
    if not args.no_e2e:
        out = np.empty(LARGE_FRAME, np.uint16)
        rec = api.Reconstructor(plan, V, LARGE_SRC, LARGE_FRAME)
        try:
            views_np = [p.numpy().view(np.uint16) for p in pinned]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rec.run(views_np, mats, IT, out)
            dt = time.perf_counter() - t0
        finally:
            rec.destroy()
        # the same transfers alone (pinned host memory, one copy per view up,
        # the result down): how much of them the pipelined run hides
        dev_buf = torch.empty((d, h, w), dtype=torch.int16, device="cuda")
        res_host = torch.empty((td, th, tw), dtype=torch.int16, pin_memory=True)
        res_dev = torch.empty((td, th, tw), dtype=torch.int16, device="cuda")
        c0, c1, c2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        c0.record()
        for v in range(V):
            dev_buf.copy_(pinned[v], non_blocking=True)
        c1.record()
        res_host.copy_(res_dev, non_blocking=True)
        c2.record()
        torch.cuda.synchronize()
        t_h2d, t_d2h = c0.elapsed_time(c1) / 1e3, c1.elapsed_time(c2) / 1e3
        del dev_buf, res_dev, res_host
        t_dev = t_total / args.steps
        e2e = {"value": voxel_iters / dt, "unit": UNIT, "ms_per_step": dt * 1e3,
               "h2d_bytes_per_step": V * d * h * w * 2, "d2h_bytes_per_step": td * th * tw * 2,
               "api": "fmvd_b200_reconstruct_host (pinned sources in, result to host memory)",
               "copies_alone_ms": {"h2d": t_h2d * 1e3, "d2h": t_d2h * 1e3},
               "hidden_fraction_of_copies": max(0.0, min(1.0, (t_dev + t_h2d + t_d2h - dt) / (t_h2d + t_d2h)))}
    cpu = cpu_baseline(frames_cpu, weights, psfs, iterations=1) if frames_cpu is not None else None
    plan.destroy()
    print(json.dumps({
        "metric": METRIC, "value": voxel_iters * args.steps / t_total, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": LARGE_NAME, "views": V, "frame": list(LARGE_FRAME), "iterations": IT,
                   "fft_plane": [H, W], "pairs_per_batch": plan.pairs_per_batch,
                   "l2": "inputs larger than L2 (77 GB resident on the device)",
                   "rl_ms_per_step": t_rl / args.steps * 1e3, "transform_ms_per_step": t_tr / args.steps * 1e3,
                   "data_generation_s": t_data},
        "roofline": {"bound": "hbm", "achieved": alg / t_rl / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / t_rl / 1e9 / peak, "peak_kind": peak_kind,
                     "kernel": "fused RL view update (line engine, 2560 x 2560 planes)",
                     "algorithmic_bytes": "14 B per padded voxel per view per iteration", "traffic": None},
        "transform": {"ms_per_step": t_tr / args.steps * 1e3, "GB_per_s": tr_bytes / t_tr / 1e9,
                      "frac_of_hbm": tr_bytes / t_tr / 1e9 / peak,
                      "algorithmic_bytes": "source read once (2 B/voxel) + frame written once (2 B/voxel)"},
        "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clk.summary(),
        "warmstart": warm,
    }), flush=True)


def large_warmstart(args, plan, frame_dev):
    """Learned warm start + RL against plain RL-50 on the large configuration's
    2048 x 2048 planes (6 views, 63 x 63 PSFs, transformed-mask weights).

    The network (6 views + their mean in, BF16 tcgen05 kernels) is trained on
    the 512 x 512 tiles of registered frame planes (a 4 x 4 grid) with targets
    = the same tiles of the planes' plain RL results (--large-target-iterations
    iterations, fewer than 50 so that a few RL iterations after the warm
    start reach the RL-50 result); at inference it runs on the same tiling of
    whole planes, and RL-k continues from the stitched estimate.  k is tuned
    on held-out planes, and both paths are timed on test planes; training,
    tuning and test planes are disjoint plane ranges of the frame."""
    import torch
    from gpu_deconvolution_b200 import warmstart as WS
    V, td, th, tw = frame_dev.shape
    N_RL, TOL, CROP = LARGE_ITERATIONS, 1e-2, 512
    n_train = args.large_train_planes
    target_its = args.large_target_iterations
    z_train = 64
    z_tune, z_test = z_train + n_train + 8, z_train + n_train + 40
    t0 = time.perf_counter()
    targets = torch.empty((n_train, th, tw), dtype=torch.float32, device="cuda")
    for z0 in range(0, n_train, 16):
        n = min(16, n_train - z0)
        est, _ = WS.rl_planes(plan, frame_dev[:, z_train + z0:z_train + z0 + n], target_its)
        targets[z0:z0 + n] = est
    # 512 x 512 crops on a 4 x 4 grid of every training plane
    cv, ct = [], []
    for y0 in range(0, th, CROP):
        for x0 in range(0, tw, CROP):
            cv.append(frame_dev[:, z_train:z_train + n_train, y0:y0 + CROP, x0:x0 + CROP])
            ct.append(targets[:, y0:y0 + CROP, x0:x0 + CROP])
    crop_views = torch.cat(cv, dim=1).contiguous()
    crop_targets = torch.cat(ct, dim=0).contiguous()
    del cv, ct, targets
    t_data = time.perf_counter() - t0
    net = WS.WarmStartNet(CROP, CROP, V, max_batch=16, seed=0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    hist = WS.train(net, crop_views, crop_targets, epochs=args.large_epochs, batch=16, lr=1e-3)
    e1.record()
    torch.cuda.synchronize()
    t_train = e0.elapsed_time(e1) / 1e3
    n_crops = crop_views.shape[1]
    del crop_views, crop_targets
    torch.cuda.empty_cache()
    # inference on the same 512 x 512 tiling as the training crops (the
    # network normalises its input per tile, so tiles must match training)
    ny, nx = th // CROP, tw // CROP

    def tiled_guess(views):
        Vv, N = views.shape[:2]
        tiles = views.reshape(Vv, N, ny, CROP, nx, CROP).permute(0, 1, 2, 4, 3, 5).reshape(Vv, N * ny * nx, CROP, CROP)
        g = net.forward(tiles.contiguous())
        return g.reshape(N, ny, nx, CROP, CROP).permute(0, 1, 3, 2, 4).reshape(N, th, tw).contiguous()

    def warm(views, k):
        guess = tiled_guess(views)
        init = torch.empty((views.shape[1], plan.fftH, plan.fftW), dtype=torch.float32, device="cuda")
        plan.pad_estimate(guess, init, 1.0)
        est, _ = WS.rl_planes(plan, views, k, init=init)
        return est

    # how well the network fits its own training targets (8 training planes)
    fit_views = frame_dev[:, z_train:z_train + 8].contiguous()
    fit_ref, _ = WS.rl_planes(plan, fit_views, target_its)
    fit_err = WS.rel_l2_planes(tiled_guess(fit_views), fit_ref.contiguous())
    tune_views = frame_dev[:, z_tune:z_tune + 8].contiguous()
    test_views = frame_dev[:, z_test:z_test + 16].contiguous()
    tune_ref, _ = WS.rl_planes(plan, tune_views, N_RL)
    tune_ref = tune_ref.contiguous()
    k, k_errors = None, {}
    for cand in tuple(range(0, 13)) + (14, 16, 20, 25, 30, 40):
        err = float(np.max(WS.rel_l2_planes(warm(tune_views, cand).contiguous(), tune_ref)))
        k_errors[cand] = err
        if err <= K_TUNE_MARGIN * TOL:
            k = cand
            break
    kk = k if k is not None else N_RL
    t_plain = WS.time_cuda(lambda: WS.rl_planes(plan, test_views, N_RL))
    t_warm = WS.time_cuda(lambda: warm(test_views, kk))
    t_net = WS.time_cuda(lambda: tiled_guess(test_views))
    warm_est = warm(test_views, kk)
    plain, _ = WS.rl_planes(plan, test_views, N_RL)
    err = WS.rel_l2_planes(warm_est.contiguous(), plain.contiguous())
    net.check()
    net.destroy()
    return {"metric": "time to the plain RL-50 result, warm start vs plain", "unit": "ms per 16 planes",
            "value": t_warm, "plain_rl50_ms": t_plain, "speedup": t_plain / t_warm, "k": k,
            "rel_l2_vs_rl50": {"max": float(err.max()), "mean": float(err.mean()), "tolerance": TOL},
            "k_search": {str(a): b for a, b in k_errors.items()}, "network_ms_per_16_planes": t_net,
            "network_vs_training_targets_rel_l2": float(np.max(fit_err)),
            "training": {"planes": n_train, "crops": n_crops, "crop": CROP, "epochs": args.large_epochs,
                         "target_rl_iterations": target_its,
                         "seconds": t_train, "loss_per_epoch": hist, "data_seconds": t_data},
            "planes": {"train": [z_train, z_train + n_train], "tune": [z_tune, z_tune + 8],
                       "test": [z_test, z_test + 16]},
            "note": "no PSNR: the frame's ground truth is not resampled"}


def run_planes(args):
    """Plain RL on square planes of the given data sizes (4 views, 10
    iterations, synthetic uint16 views), one JSON line per size: padded
    voxel-view-iterations per second (padded plane x planes x views x
    iterations over the CUDA-event time of DevicePlan.run)."""
    import torch
    import numpy as np
    from gpu_deconvolution_b200 import api, synth
    V, IT = 4, 2 if args.small else 10
    for size in [int(x) for x in args.planes.split(",") if x]:
        k = 63 if size >= 2000 else 31
        psfs = [synth.gaussian_psf(k, k, 1.2, 5.0, 45.0 * v) for v in range(V)]
        weights = [np.ones((size, size), np.float32) for _ in range(V)]
        plan = api.DevicePlan(size, size, weights, [q.copy() for q in psfs], 0,
                              pairs_per_batch=args.pairs_per_batch)
        fh, fw = plan.fftH, plan.fftW
        D = 8 if args.small else max(8, 2 * int(96e6 // (fh * fw * 8)) * 2)
        g = torch.Generator(device="cuda").manual_seed(size)
        views = torch.randint(100, 3000, (V, D, size, size), dtype=torch.int32, device="cuda", generator=g)
        views = views.to(torch.int16)
        out = torch.zeros((D, size, size), dtype=torch.int16, device="cuda")
        for _ in range(max(1, args.warmup)):
            plan.run(views, out, IT)
        torch.cuda.synchronize()
        ts = []
        for _ in range(max(1, args.steps)):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            plan.run(views, out, IT)
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        ms = float(np.median(ts))
        print(json.dumps({"metric": "padded voxel-view-iter/s", "value": fh * fw * D * V * IT / (ms * 1e-3),
                          "unit": "voxel-view-iter/s", "ms": ms, "higher_is_better": True, "dtype": "f32",
                          "data": "synthetic",
                          "config": {"workload": f"plain RL, {V} views, {IT} iterations, {D} planes of "
                                                 f"{size} x {size} ({k} x {k} PSFs)", "fft_plane": [fh, fw],
                                     "pairs_per_batch": plan.pairs_per_batch}}), flush=True)
        plan.destroy()
        del views, out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "warmstart":
        run_warmstart(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "planes":
        run_planes(args)
    elif args.workload == "large":
        run_large(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
