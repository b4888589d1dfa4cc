"""Host-buffer reconstruction (fmvd_b200_reconstruct_host): resampling and
plain RL with the frame kept on the device must give exactly the result of
the device-resident steps (transform_device for every view, then
DevicePlan.run), for chunked and single-chunk runs, pageable and pinned
sources, and on repeated calls."""
import numpy as np
import pytest

from gpu_deconvolution_b200 import api, synth

pytestmark = pytest.mark.gpu


def _case(bits=16, seed=5):
    rng = np.random.default_rng(seed)
    src = (12, 40, 48)
    frame = (30, 48, 64)
    V = 2
    hi = 4000 if bits == 16 else 200
    dt = np.uint16 if bits == 16 else np.uint8
    views = [rng.integers(0, hi, src).astype(dt) for _ in range(V)]
    mats = [synth.rotation_y_inverse(90.0 * v + 5.0, frame, src, 2.5, (0.4 * v, -0.3, 0.2)) for v in range(V)]
    psfs = [synth.gaussian_psf(9, 9, 1.0, 2.2, 70.0 * v) for v in range(V)]
    rng2 = np.random.default_rng(seed + 1)
    weights = [rng2.uniform(0.5, 1.5, frame[1:]).astype(np.float32) for _ in range(V)]
    return views, mats, psfs, weights, src, frame


def _device_reference(plan, views, mats, src, frame, iterations, bits):
    import torch
    d, h, w = src
    td, th, tw = frame
    V = len(views)
    pitch = api.source_pitch(bits, w)
    dt = torch.int16 if bits == 16 else torch.uint8
    npdt = np.int16 if bits == 16 else np.uint8
    fr = torch.zeros((V, td, th, tw), dtype=dt, device="cuda")
    for v in range(V):
        s = torch.zeros((d, h, pitch), dtype=dt, device="cuda")
        s[:, :, :w] = torch.from_numpy(views[v].view(npdt)).cuda()
        api.transform_device(s, pitch, w, h, d, mats[v], tw, th, 0, td, out=fr[v], bits=bits)
    out = torch.zeros((td, th, tw), dtype=dt, device="cuda")
    plan.run(fr, out, iterations)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint16 if bits == 16 else np.uint8)


@pytest.mark.parametrize("bits,chunk", [(16, 8), (16, 0), (8, 7)])
def test_reconstruct_host_matches_device_steps(bits, chunk):
    import torch
    views, mats, psfs, weights, src, frame = _case(bits)
    td, th, tw = frame
    plan = api.DevicePlan(th, tw, weights, [p.copy() for p in psfs], 0, bits=bits, pairs_per_batch=2)
    try:
        ref = _device_reference(plan, views, mats, src, frame, 4, bits)
        rec = api.Reconstructor(plan, len(views), src, frame, chunk)
        try:
            out1 = rec.run(views, mats, 4)
            pinned = [torch.from_numpy(v.view(np.int16 if bits == 16 else np.uint8)).pin_memory().numpy()
                      .view(v.dtype) for v in views]
            out2 = rec.run(pinned, mats, 4)
        finally:
            rec.destroy()
        np.testing.assert_array_equal(out1, ref)
        np.testing.assert_array_equal(out2, ref)
        assert out1.any()
    finally:
        plan.destroy()
