"""Plane sharding of one multi-view volume over the ranks of a job.

Richardson-Lucy in the reference is strictly plane-wise
(fmvd_deconvolve.impl.cpp:205-300 streams z-planes independently; kernels and
weights are 2-D), and the resampler computes every target plane on its own
(fmvd_transform.impl.cu:120-128).  So a volume splits into contiguous
target-plane ranges, one per rank, with no exchange between ranks:

* every rank holds the (small) kernel spectra and weight images;
* every rank uploads only the source planes its target planes sample
  (``source_planes``) into its own GPU memory and resamples its range;
* every rank deconvolves its planes and writes them at their offset of the
  result file (``write_planes``) or hands them to rank 0 (``gather_planes``).

The result is identical to a single-GPU run of the whole volume: each output
plane goes through the same kernels with the same inputs.
"""
from __future__ import annotations

import math
import os

import numpy as np


def plane_range(n_planes: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [z0, z1) of ``n_planes`` for ``rank`` of ``world``;
    the first ``n_planes % world`` ranks take one plane more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n_planes < 0:
        raise ValueError("negative plane count")
    base, extra = divmod(n_planes, world)
    z0 = rank * base + min(rank, extra)
    return z0, z0 + base + (1 if rank < extra else 0)


def source_planes(inverse, w: int, h: int, d: int, tw: int, th: int, z0: int, z1: int) -> tuple[int, int]:
    """Source planes [s0, s1) that target planes [z0, z1) of a tw x th frame
    read through the 3x4 target->source matrix ``inverse``
    (fmvd_transform.impl.cu:24-56: source z = row 2 of the matrix applied to
    (x, y, z, 1), sampled trilinearly at z + 0.5, so planes floor(z) and
    floor(z) + 1 carry weight).  The affine map reaches its extremes at the
    corners of the target box; one plane of margin each side absorbs float
    rounding.  Returns (0, 0) when no source plane is read."""
    if z1 <= z0:
        return 0, 0
    m = np.asarray(inverse, np.float64).reshape(3, 4)
    zs = [m[2, 0] * x + m[2, 1] * y + m[2, 2] * z + m[2, 3]
          for x in (0, tw - 1) for y in (0, th - 1) for z in (z0, z1 - 1)]
    lo = math.floor(min(zs)) - 1
    hi = math.floor(max(zs)) + 2
    s0, s1 = max(lo, 0), min(hi + 1, d)
    return (s0, s1) if s1 > s0 else (0, 0)


def write_planes(path: str, planes: np.ndarray, z0: int) -> None:
    """Write ``planes`` (n x th x tw samples) at plane offset ``z0`` of the
    raw z-major result file ``path`` (the reference's on-disk layout,
    fmvd_deconvolve_hdd.impl.cpp:16-34).  The file is created if missing and
    never truncated, so ranks can write their ranges in any order."""
    planes = np.ascontiguousarray(planes)
    plane_bytes = planes[0].nbytes if planes.shape[0] else 0
    fd = os.open(path, os.O_WRONLY | os.O_CREAT, 0o644)
    try:
        data = memoryview(planes.reshape(-1).view(np.uint8))
        off, pos = z0 * plane_bytes, 0
        while pos < len(data):
            pos += os.pwrite(fd, data[pos:], off + pos)
    finally:
        os.close(fd)


def gather_planes(local: np.ndarray, z0: int, n_planes: int, group=None):
    """Collects every rank's planes on rank 0 of the initialised process group
    (any backend): returns the assembled n_planes x ... volume on rank 0 and
    None elsewhere.  This only moves results; no rank waits for another
    before its own compute is done."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    items = [None] * world if rank == 0 else None
    dist.gather_object((z0, np.ascontiguousarray(local)), items, dst=0, group=group)
    if rank != 0:
        return None
    out = np.zeros((n_planes,) + local.shape[1:], local.dtype)
    for zs, block in items:
        out[zs:zs + block.shape[0]] = block
    return out


def run_shard(views, inverses, frame, kernels, weights, iterations, rank, world, psf_type=0, bits=16,
              pairs_per_batch=0, stream=None):
    """Resample and deconvolve this rank's target planes on the current CUDA
    device.

    views: list of V source volumes (d x h x w uint16/uint8, host arrays);
    inverses: V 3x4 target->source matrices; frame: (td, th, tw);
    kernels, weights, psf_type, iterations: as for ``fmvd_initialize_cuda_*``.
    Returns (z0, planes) with planes the rank's (z1 - z0) x th x tw result on
    the host.  Only the source planes the range samples are copied to the
    device; the rest of the source buffer is zero and never weighted.
    """
    import torch

    from . import api

    td, th, tw = frame
    z0, z1 = plane_range(td, rank, world)
    dtype = torch.int16 if bits == 16 else torch.uint8
    npdt = np.int16 if bits == 16 else np.uint8
    n = z1 - z0
    out = np.zeros((n, th, tw), np.uint16 if bits == 16 else np.uint8)
    if n == 0:
        return z0, out
    V = len(views)
    d, h, w = views[0].shape
    pitch = api.source_pitch(bits, w)
    s = stream if stream is not None else torch.cuda.current_stream()
    with torch.cuda.stream(s):
        src = torch.zeros((d, h, pitch), dtype=dtype, device="cuda")
        frame_dev = torch.empty((V, n, th, tw), dtype=dtype, device="cuda")
        for v in range(V):
            s0, s1 = source_planes(inverses[v], w, h, d, tw, th, z0, z1)
            src.zero_()
            if s1 > s0:
                slab = np.ascontiguousarray(views[v][s0:s1]).view(npdt)
                src[s0:s1, :, :w].copy_(torch.from_numpy(slab).pin_memory(), non_blocking=True)
            api.transform_device(src, pitch, w, h, d, inverses[v], tw, th, z0, n, out=frame_dev[v],
                                 stream=s.cuda_stream, bits=bits)
        res = torch.empty((n, th, tw), dtype=dtype, device="cuda")
        plan = api.DevicePlan(th, tw, weights, [np.array(k, np.float32) for k in kernels], psf_type, bits=bits,
                              pairs_per_batch=pairs_per_batch)
        try:
            plan.run(frame_dev, res, iterations, stream=s.cuda_stream)
            host = res.cpu()
        finally:
            plan.destroy()
    out[...] = host.numpy().view(out.dtype)
    return z0, out
