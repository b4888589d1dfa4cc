"""Plane sharding of one volume over ranks (gpu_deconvolution_b200.shard).

CPU tests check the host logic: the plane partition, that the source slab a
rank uploads holds every plane its target planes weight (planes outside the
slab are overwritten with a sentinel and the oracle's resampling must not
change), and gloo jobs of two and three ranks whose ranks each run
``shard.run_shard`` (plane range, source slabs, result offsets) with the
oracle standing in for the device resampler and RL, write their planes to one
file and hand them to rank 0; both must match a single-process run of the
whole volume.  The GPU test runs the same splits through the native library.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

from conftest import ROOT
from gpu_deconvolution_b200 import shard, synth
from oracle import fmvd_oracle as O


def small_case(seed=3, bits=16):
    rng = np.random.default_rng(seed)
    src = (10, 24, 20)  # d, h, w
    frame = (20, 24, 20)  # td, th, tw
    V = 2
    maxv = (1 << bits) - 1
    views = [rng.integers(0, maxv // 4, src).astype(np.uint16 if bits == 16 else np.uint8) for _ in range(V)]
    mats = [synth.rotation_y_inverse(90.0 * v + 7.0, frame, src, 2.0, (0.3 * v, -0.2, 0.4)) for v in range(V)]
    psfs = [synth.gaussian_psf(5, 5, 1.0, 1.6, 30.0 * v) for v in range(V)]
    weights = [np.ones(frame[1:], np.float32) for _ in range(V)]
    return views, mats, psfs, weights, src, frame


def test_plane_range_partition():
    for n in (0, 1, 5, 17, 384):
        for world in (1, 2, 3, 4, 8):
            ranges = [shard.plane_range(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            for (a0, a1), (b0, b1) in zip(ranges, ranges[1:]):
                assert a1 == b0
            pairs = [(b - a + 1) // 2 for a, b in ranges]
            assert max(pairs) - min(pairs) <= 1 and min(pairs) >= 0
            # every share starts at an even plane (plane pairs stay together)
            assert all(a % 2 == 0 for a, b in ranges if b > a)
    with pytest.raises(ValueError):
        shard.plane_range(4, 2, 2)


@pytest.mark.parametrize("world", [2, 3, 5])
def test_source_slab_holds_every_weighted_plane(world):
    views, mats, _, _, src, frame = small_case()
    d, h, w = src
    td, th, tw = frame
    for v in range(len(views)):
        full = O.transform_volume(views[v], mats[v], td, th, tw)
        for r in range(world):
            z0, z1 = shard.plane_range(td, r, world)
            s0, s1 = shard.source_planes(mats[v], w, h, d, tw, th, z0, z1)
            poisoned = views[v].copy()
            poisoned[:s0] = 65535
            poisoned[s1:] = 65535
            part = O.transform_volume(poisoned, mats[v], td, th, tw)[z0:z1]
            np.testing.assert_array_equal(part, full[z0:z1])
            if world > 2 and v == 0:
                assert s1 - s0 < d  # near-axial view: the slab is a strict part of the source


def test_source_slab_outside_source_is_empty():
    m = np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 100], np.float32)
    assert shard.source_planes(m, 8, 8, 10, 8, 8, 0, 4) == (0, 0)
    assert shard.source_planes(m, 8, 8, 10, 8, 8, 3, 3) == (0, 0)


def test_write_planes_any_order():
    planes = np.arange(5 * 3 * 4, dtype=np.uint16).reshape(5, 3, 4)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "out.raw")
        shard.write_planes(path, planes[3:], 3)
        shard.write_planes(path, planes[:3], 0)
        back = np.fromfile(path, np.uint16).reshape(5, 3, 4)
    np.testing.assert_array_equal(back, planes)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_resample(frame):
    td, th, tw = frame

    def resample(v, slab, s0, inverse, z0, n):
        # only the slab is known to the rank: the rest of the source is zero
        vol = np.zeros(_SRC_SHAPE, slab.dtype)
        vol[s0:s0 + slab.shape[0]] = slab
        return O.transform_volume(vol, inverse, td, th, tw)[z0:z0 + n]
    return resample


def _oracle_deconvolve(psfs, weights, iterations):
    return lambda frames: O.deconvolve_volume(np.stack(frames), weights, psfs, 0, iterations)


_SRC_SHAPE = small_case()[4]


def _gloo_rank(rank, world, port, outfile, result):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from gpu_deconvolution_b200 import shard as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        views, mats, psfs, weights, src, frame = small_case()
        # the library's host logic (plane range, source slabs, offsets) with
        # the oracle standing in for the device resampler and RL
        z0, local = S.run_shard(views, mats, frame, psfs, weights, 3, rank, world,
                                resample=_oracle_resample(frame), deconvolve=_oracle_deconvolve(psfs, weights, 3))
        assert (z0, z0 + local.shape[0]) == S.plane_range(frame[0], rank, world)
        S.write_planes(outfile, local, z0)
        full = S.gather_planes(local, z0, frame[0])
        if rank == 0:
            np.save(result, full)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_job_matches_single_process(world):
    """A world-rank gloo job (world 3 splits 20 planes as 8 + 6 + 6) through
    run_shard's host logic matches one process running the whole volume."""
    import torch.multiprocessing as mp
    views, mats, psfs, weights, src, frame = small_case()
    td, th, tw = frame
    resampled = np.stack([O.transform_volume(views[v], mats[v], td, th, tw) for v in range(len(views))])
    expect = O.deconvolve_volume(resampled, weights, psfs, 0, 3)
    with tempfile.TemporaryDirectory() as tmp:
        outfile = os.path.join(tmp, "result.raw")
        result = os.path.join(tmp, "gathered.npy")
        mp.start_processes(_gloo_rank, args=(world, _free_port(), outfile, result), nprocs=world, join=True,
                           start_method="spawn")
        gathered = np.load(result)
        written = np.fromfile(outfile, np.uint16).reshape(td, th, tw)
    np.testing.assert_array_equal(gathered, expect)
    np.testing.assert_array_equal(written, expect)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_run_matches_whole_volume_gpu(world):
    """Ranks of a split run one after another on one GPU (they never wait on
    each other); shares start at even planes, so each plane keeps its
    partner in the paired FFT and the assembled volume is bit-identical to
    the whole-volume run (world 3: an uneven 8 + 6 + 6 split)."""
    views, mats, psfs, weights, src, frame = small_case()
    td = frame[0]
    _, whole = shard.run_shard(views, mats, frame, psfs, weights, 4, 0, 1)
    parts = [shard.run_shard(views, mats, frame, psfs, weights, 4, r, world) for r in range(world)]
    assert all(z0 % 2 == 0 for z0, _ in parts)
    assembled = np.concatenate([p for _, p in parts])
    assert assembled.shape[0] == td
    np.testing.assert_array_equal(assembled, whole)
