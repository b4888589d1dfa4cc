"""fmvd_b200_deconvolve_device_noalloc against fmvd_b200_deconvolve_device.

Both entry points are called through the C ABI on the same plan and inputs.
The no-allocation call runs twice in a row on different inputs, so a result
that leaned on the previous call's contents of the shared work array would
show up in the second comparison.  This file is collected last and also
passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2
from gpu_deconvolution_b200 import api, native, synth

pytestmark = pytest.mark.gpu


def _views(torch, V, D, H, W, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randint(50, 4000, (V, D, H, W), dtype=torch.int32, device="cuda", generator=g).to(torch.int16)


def _run(lib, entry, plan, views, iterations, fftH, fftW):
    torch = pytest.importorskip("torch")
    V, D, H, W = views.shape
    out = torch.zeros((D, H, W), dtype=torch.int16, device="cuda")
    est = torch.zeros((D, fftH, fftW), dtype=torch.float32, device="cuda")
    native.clear_errors()
    r = getattr(lib, entry)(plan.plan, views.data_ptr(), D * H * W, out.data_ptr(), D, iterations, est.data_ptr(),
                            None)
    native.check(entry)
    assert r == 0
    torch.cuda.synchronize()
    assert lib.fmvd_b200_plan_check(plan.plan) == 0
    return out.cpu().numpy().view(np.uint16), est.cpu().numpy()


@pytest.mark.parametrize("pairs", [1, 2])
def test_noalloc_matches_plan_entry_two_calls(pairs):
    torch = pytest.importorskip("torch")
    lib = native.load()
    H, W, V, D, iters = 200, 184, 3, 7, 4
    psfs = [synth.gaussian_psf(9, 9, 1.0, 2.5, 60.0 * v) for v in range(V)]
    weights = [np.full((H, W), 1.0 + v, np.float32) for v in range(V)]
    plan = api.DevicePlan(H, W, weights, psfs, 0, bits=16, pairs_per_batch=pairs)
    try:
        for call, seed in enumerate((11, 12)):
            views = _views(torch, V, D, H, W, seed)
            ref_out, ref_est = _run(lib, "fmvd_b200_deconvolve_device", plan, views, iters, plan.fftH, plan.fftW)
            out, est = _run(lib, "fmvd_b200_deconvolve_device_noalloc", plan, views, iters, plan.fftH, plan.fftW)
            # same kernels and batch split: expected bit-identical; tolerance
            # 1e-6 relative L2 on the estimate, one sample unit on the output
            assert rel_l2(est, ref_est) < 1e-6, f"call {call}"
            assert int(np.abs(out.astype(np.int64) - ref_out.astype(np.int64)).max()) <= 1, f"call {call}"
    finally:
        plan.destroy()


def test_noalloc_several_batches_fewer_pairs_than_plan():
    """1024 x 1024 padded planes: the shared array holds 3 plane pairs, the
    plan's batch 8, so 11 planes run as two batches in the array, at a batch
    size the plan itself never uses."""
    torch = pytest.importorskip("torch")
    lib = native.load()
    H = W = 1000
    V, D, iters = 2, 11, 2
    psfs = [synth.gaussian_psf(9, 9, 1.0, 2.0, 90.0 * v) for v in range(V)]
    weights = [np.full((H, W), 1.0, np.float32) for _ in range(V)]
    plan = api.DevicePlan(H, W, weights, psfs, 0, bits=16, pairs_per_batch=8)
    try:
        assert (plan.fftH, plan.fftW, plan.pairs_per_batch) == (1024, 1024, 8)
        for call, seed in enumerate((21, 22)):
            views = _views(torch, V, D, H, W, seed)
            ref_out, ref_est = _run(lib, "fmvd_b200_deconvolve_device", plan, views, iters, plan.fftH, plan.fftW)
            out, est = _run(lib, "fmvd_b200_deconvolve_device_noalloc", plan, views, iters, plan.fftH, plan.fftW)
            # batch size changes only the schedule, so this too is expected to
            # match bit for bit; same tolerances as above
            assert rel_l2(est, ref_est) < 1e-6, f"call {call}"
            assert int(np.abs(out.astype(np.int64) - ref_out.astype(np.int64)).max()) <= 1, f"call {call}"
    finally:
        plan.destroy()


def test_noalloc_rejects_plane_beyond_array():
    lib = native.load()
    H = W = 2000  # padded plane 2048 x 2048: one plane pair needs 64 MiB of work memory
    plan = api.DevicePlan(H, W, [np.ones((H, W), np.float32)], [synth.gaussian_psf(3, 3, 1.0, 1.0, 0.0)], 0,
                          bits=16, pairs_per_batch=1)
    try:
        assert (plan.fftH, plan.fftW) == (2048, 2048)
        native.clear_errors()
        r = lib.fmvd_b200_deconvolve_device_noalloc(plan.plan, None, 0, None, 1, 1, None, None)
        assert r != 0
        with pytest.raises(native.FmvdError, match="more than its fixed"):
            native.check("fmvd_b200_deconvolve_device_noalloc")
    finally:
        native.clear_errors()
        plan.destroy()
