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
    """Contiguous share [z0, z1) of ``n_planes`` for ``rank`` of ``world``.

    Planes are dealt in pairs (2p, 2p + 1), the pairs the library packs into
    one complex transform, so every share starts at an even plane and each
    plane keeps the partner it has in a whole-volume run: the assembled
    result is then bit-identical to one GPU deconvolving the whole volume.
    The first ``n_pairs % world`` ranks take one pair more; only the last
    non-empty share can end on an unpaired plane (when ``n_planes`` is odd)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n_planes < 0:
        raise ValueError("negative plane count")
    pairs = (n_planes + 1) // 2
    base, extra = divmod(pairs, world)
    p0 = rank * base + min(rank, extra)
    p1 = p0 + base + (1 if rank < extra else 0)
    return min(2 * p0, n_planes), min(2 * p1, n_planes)


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
              pairs_per_batch=0, stream=None, resample=None, deconvolve=None):
    """Resample and deconvolve this rank's target planes.

    views: list of V source volumes (d x h x w uint16/uint8, host arrays);
    inverses: V 3x4 target->source matrices; frame: (td, th, tw);
    kernels, weights, psf_type, iterations: as for ``fmvd_initialize_cuda_*``.
    Returns (z0, planes) with planes the rank's (z1 - z0) x th x tw result on
    the host.  Only the source planes the range samples are handed on; the
    rest of each source volume is zero and never weighted.

    ``resample(v, slab, s0, inverse, z0, n)`` (slab: source planes
    [s0, s0 + len(slab)) of view v) returns the resampled frame planes
    [z0, z0 + n) of that view, and ``deconvolve(frames)`` (V x n x th x tw)
    returns the n result planes; by default both run on the current CUDA
    device through the native library (``DeviceShard``)."""
    td, th, tw = frame
    z0, z1 = plane_range(td, rank, world)
    n = z1 - z0
    out = np.zeros((n, th, tw), np.uint16 if bits == 16 else np.uint8)
    if n == 0:
        return z0, out
    V = len(views)
    d, h, w = views[0].shape
    dev = None
    if resample is None or deconvolve is None:
        dev = DeviceShard(views[0].shape, frame, n, V, kernels, weights, psf_type, bits, pairs_per_batch, iterations,
                          stream)
        resample = resample or dev.resample
        deconvolve = deconvolve or dev.deconvolve
    try:
        frames = []
        for v in range(V):
            s0, s1 = source_planes(inverses[v], w, h, d, tw, th, z0, z1)
            frames.append(resample(v, views[v][s0:s1], s0, inverses[v], z0, n))
        out[...] = deconvolve(frames)
    finally:
        if dev is not None:
            dev.destroy()
    return z0, out


class DeviceShard:
    """The device half of ``run_shard``: a source buffer the size of one view
    (only the slab is copied in), the rank's resampled frame and a plan, on
    the current CUDA device and ``stream``."""

    def __init__(self, src_shape, frame, n, V, kernels, weights, psf_type, bits, pairs_per_batch, iterations,
                 stream=None):
        import torch

        from . import api
        self.api = api
        self.bits = bits
        self.iterations = iterations
        self.dtype = torch.int16 if bits == 16 else torch.uint8
        self.npdt = np.int16 if bits == 16 else np.uint8
        d, h, w = src_shape
        td, th, tw = frame
        self.src_shape, self.frame, self.n = src_shape, frame, n
        self.pitch = api.source_pitch(bits, w)
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        self.src = torch.zeros((d, h, self.pitch), dtype=self.dtype, device="cuda")
        self.frame_dev = torch.empty((V, n, th, tw), dtype=self.dtype, device="cuda")
        self.res = torch.empty((n, th, tw), dtype=self.dtype, device="cuda")
        self.plan = api.DevicePlan(th, tw, weights, [np.array(k, np.float32) for k in kernels], psf_type, bits=bits,
                                   pairs_per_batch=pairs_per_batch)

    def resample(self, v, slab, s0, inverse, z0, n):
        import torch
        d, h, w = self.src_shape
        td, th, tw = self.frame
        with torch.cuda.stream(self.stream):
            self.src.zero_()
            if slab.shape[0]:
                host = torch.from_numpy(np.ascontiguousarray(slab).view(self.npdt)).pin_memory()
                self.src[s0:s0 + slab.shape[0], :, :w].copy_(host, non_blocking=True)
            self.api.transform_device(self.src, self.pitch, w, h, d, inverse, tw, th, z0, n, out=self.frame_dev[v],
                                      stream=self.stream.cuda_stream, bits=self.bits)
        return self.frame_dev[v]

    def deconvolve(self, frames):
        import torch
        with torch.cuda.stream(self.stream):
            self.plan.run(self.frame_dev, self.res, self.iterations, stream=self.stream.cuda_stream)
            host = self.res.cpu()
        return host.numpy().view(np.uint16 if self.bits == 16 else np.uint8)

    def destroy(self):
        if self.plan is not None:
            self.plan.destroy()
            self.plan = None
