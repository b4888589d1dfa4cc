"""Parity at each configuration's own geometry and iteration depth, against
both the reference's CUDA build and the FP64 oracle.

For every case the same views, weights and kernels go through
* this library (``DevicePlan.run`` through the C ABI; float estimate on the
  FFT plane after k iterations),
* the reference library built from the upstream sources
  (oracle/_ref/libfmvd_ref.so: fmvd_initialize / deconvolve_planes / destroy
  with nstreams 1, the float estimate read from the plan in the datasink;
  the loop it runs is fmvd_deconvolve.impl.cpp:262-273), and
* the FP64 oracle (oracle/fmvd_oracle.py), run once with a snapshot of the
  estimate after each checked iteration count.

Tolerance: 1e-4 relative L2 per checked iteration count, against the
reference build and against the oracle; sample outputs
within one unit of the reference build.  Cases:
* plain RL, small: 2 views, 256 x 256 data, 17 x 17 PSFs, 10 iterations,
  4 planes (FFT plane 512 x 512);
* transform + plain RL plane: 4 views, 512 x 512 data, 31 x 31 rotated PSFs,
  transformed-mask weights, 20 iterations (FFT plane 1024 x 1024);
* large planes: 1400 x 1400 (FFT 1536) and 2048 x 2048 (FFT 2560) data with
  63 x 63 PSFs, 4 views, 10 iterations.
Two planes per large case, so both halves of a packed plane pair are checked.
"""
import multiprocessing as mp

import numpy as np
import pytest

from conftest import rel_l2
from gpu_deconvolution_b200 import api, synth
from oracle import fmvd_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _oracle_plane(args):
    """FP64 oracle estimates of one plane after each count in ``checks``."""
    H, W, weights, kernels, psf, planes, checks = args
    plan = O.Plan(H, W, list(weights), list(kernels), psf)
    pv = [plan.pad_data(p) for p in planes]
    e = plan.initial_estimate()
    done, out = 0, {}
    for k in sorted(checks):
        e = plan.iterate(e, pv, k - done)
        done = k
        out[k] = e
    return out


def oracle_checkpoints(views, weights, kernels, psf, checks):
    """{k: D x fftH x fftW} FP64 estimates; planes run in parallel in spawned
    processes (never forked from a process that has initialised CUDA)."""
    V, D, H, W = views.shape
    jobs = [(H, W, [np.asarray(w) for w in weights], [np.asarray(k) for k in kernels], psf,
             [views[v, z] for v in range(V)], tuple(checks)) for z in range(D)]
    with mp.get_context("spawn").Pool(min(D, 8)) as pool:
        per_plane = pool.map(_oracle_plane, jobs)
    return {k: np.stack([p[k] for p in per_plane]) for k in checks}


def library_estimate(views, weights, kernels, psf, iterations):
    import torch
    V, D, H, W = views.shape
    plan = api.DevicePlan(H, W, weights, [np.array(k, np.float32) for k in kernels], psf, bits=16)
    try:
        tv = torch.from_numpy(np.ascontiguousarray(views).view(np.int16)).cuda()
        out = torch.zeros((D, H, W), dtype=torch.int16, device="cuda")
        est = torch.zeros((D, plan.fftH, plan.fftW), dtype=torch.float32, device="cuda")
        plan.run(tv, out, iterations, est)
        torch.cuda.synchronize()
        assert plan.lib.fmvd_b200_plan_check(plan.plan) == 0
        return out.cpu().numpy().view(np.uint16), est.cpu().numpy()
    finally:
        plan.destroy()


def check_case(ref_lib, views, weights, kernels, checks, psf=0):
    from oracle import ref_lib as R
    lib, _ = ref_lib
    D = views.shape[1]
    orc = oracle_checkpoints(views, weights, kernels, psf, checks)
    report = {}
    for k in checks:
        out, est = library_estimate(views, weights, kernels, psf, k)
        ref = R.ref_deconvolve(lib, views, weights, [np.array(q, np.float32) for q in kernels], psf, k, 1, True)
        assert ref["est"].shape == est.shape
        e_ref = rel_l2(est, ref["est"])
        e_orc = rel_l2(est, orc[k])
        e_ref_orc = rel_l2(ref["est"], orc[k])
        report[k] = (e_ref, e_orc, e_ref_orc)
        assert e_ref < TOL, f"iteration {k}: rel L2 {e_ref:.3g} vs the reference build ({report})"
        assert e_orc < TOL, f"iteration {k}: rel L2 {e_orc:.3g} vs the FP64 oracle ({report})"
        d = np.abs(out.astype(np.int64) - ref["out"][:D].astype(np.int64))
        assert d.max() <= 1, f"iteration {k}: sample difference {d.max()} vs the reference build"
    print("rel L2 (library vs reference, library vs oracle, reference vs oracle):",
          {k: tuple(f"{x:.2e}" for x in v) for k, v in report.items()})
    return report


def torch_views(D, H, W, psfs, seed):
    """Bead planes blurred by each PSF with Poisson noise (uint16), on the GPU."""
    import torch
    gt, g = synth.bead_volume_torch(D, H, W, seed, "cuda", density=2e-4)
    v = synth.blur_noise_torch(gt, psfs, g)
    torch.cuda.synchronize()
    return v.cpu().numpy().view(np.uint16)


def test_plain_rl_small_full_depth(ref_lib):
    """2 views of 256 x 256, 17 x 17 PSFs (sigma 1.5 x 4.0, 0 / 90 degrees),
    equal weights, 10 iterations, 4 planes."""
    views, psfs, weights, _ = synth.plain_rl_views(shape=(4, 256, 256), n_views=2, n_beads=60, ksize=17,
                                                  sigma=(1.5, 4.0), seed=41)
    check_case(ref_lib, views, list(weights), psfs, [1, 5, 10])


def test_transform_plane_1024_full_depth(ref_lib):
    """4 views of 512 x 512, 31 x 31 PSFs (sigma 1.2 x 5.0, rotated per view),
    transformed-mask weights of the rotated views, 20 iterations."""
    V, H = 4, 512
    psfs = [synth.gaussian_psf(31, 31, 1.2, 5.0, 180.0 * v / V) for v in range(V)]
    views = torch_views(2, H, H, psfs, 43)
    frame, src = (384, H, H), (128, H, H)
    shifts = np.random.default_rng(43).uniform(-8, 8, (V, 3))
    weights = [O.transformed_mask(synth.rotation_y_inverse(90.0 * v, frame, src, 3.0, shifts[v]), 200, H, H, 128,
                                  3.0, H, H, 16.0).astype(np.float32) for v in range(V)]
    assert all(w.min() < 1e-3 and w.max() > 0.99 for w in weights)
    check_case(ref_lib, views, weights, psfs, [1, 5, 10, 20])


@pytest.mark.parametrize("size,fft", [(1400, 1536), (2048, 2560)])
def test_large_planes_63_psf(ref_lib, size, fft):
    """4 views of size x size, 63 x 63 PSFs (sigma 2 x 8, rotated per view),
    uneven weights, 10 iterations, one plane pair (line engine)."""
    V = 4
    psfs = [synth.gaussian_psf(63, 63, 2.0, 8.0, 45.0 * v) for v in range(V)]
    views = torch_views(2, size, size, psfs, size)
    rng = np.random.default_rng(size)
    weights = [rng.uniform(0.2, 1.0, (size, size)).astype(np.float32) for _ in range(V)]
    assert O.snap_transform_size(size + 62) == fft
    check_case(ref_lib, views, weights, psfs, [1, 5, 10])
