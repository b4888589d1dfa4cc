"""Resampler and weight mask on the GPU, through the C ABI, against the
hardware texture path of the reference resampler (texture-object
restatement, oracle/_ref) and against the CPU oracle.

Tolerance: against the CPU oracle (the same weight model) within one sample
unit, the final rounding of v * 2^bits + 0.5.  Against the texture unit,
whose 1/256 weight rounding differs from the model's by one step for some
coordinates, within the change one weight step per axis can make (the
oracle's transform_weight_sensitivity) plus one unit.
"""
import os

import numpy as np
import pytest

from conftest import REF_DIR
from gpu_deconvolution_b200 import api, synth
from oracle import fmvd_oracle as O

pytestmark = pytest.mark.gpu


def volume(seed=1, shape=(20, 24, 28), bits=16):
    rng = np.random.default_rng(seed)
    d, h, w = shape
    zz, yy, xx = np.meshgrid(np.arange(d), np.arange(h), np.arange(w), indexing="ij")
    v = 20000 + 15000 * np.sin(xx / 3.0) * np.cos(yy / 4.0) + 8000 * np.sin(zz / 2.5) + rng.normal(0, 2000, shape)
    v = np.clip(v, 0, 65535).astype(np.uint16)
    v[5:8, 5:8, 5:8] = 65535
    return v if bits == 16 else (v >> 8).astype(np.uint8)


def matrices(frame, src_shape):
    rng = np.random.default_rng(2)
    a = np.eye(3) + rng.normal(0, 0.15, (3, 3))
    return [
        np.array([1, 0, 0, 2.25, 0, 1, 0, -1.5, 0, 0, 1, 0.75], np.float32),
        synth.rotation_y_inverse(90.0, frame, src_shape, 2.0, (0.3, -0.7, 0.2)),
        synth.rotation_y_inverse(270.0, frame, src_shape, 3.0, (1.0, 0.5, -0.25)),
        np.concatenate([a, rng.uniform(-2, 2, (3, 1))], axis=1).astype(np.float32).reshape(-1),
    ]


def check_samples(got, ref):
    """Same weight model (the CPU oracle): equal up to the final rounding."""
    d = np.abs(got.astype(np.int64) - ref.astype(np.int64))
    assert d.max() <= 1, d.max()
    assert (d > 0).mean() < 2e-2


def check_vs_texture_unit(got, ref, src, m, frame, bits):
    """Against the hardware texture path: within one 1/256 weight step per
    axis (the unit's weight granularity), plus one unit of rounding."""
    bits_max = (1 << bits) - 1
    sens = O.transform_weight_sensitivity(src, m, *frame, bits=bits)
    d = np.abs(got.astype(np.int64) - ref.astype(np.int64))
    d = np.minimum(d, bits_max + 1 - d)  # 0 and 2^bits - 1 are one wrap apart
    assert np.all(d <= sens + 1), (d - sens).max()
    if bits == 8:
        # one 8-bit unit is 256 16-bit units: the weight rounding rarely shows
        assert (d == 0).mean() > 0.5


@pytest.mark.parametrize("bits", [16, 8])
@pytest.mark.parametrize("mi", [0, 1, 2, 3])
def test_transform_vs_oracle(bits, mi):
    src = volume(bits=bits)
    frame = (24, 20, 28)
    m = matrices(frame, src.shape)[mi]
    got = api.transform_host(src, m, frame[2], frame[1], frame[0])
    ref = O.transform_volume(src, m, *frame, bits=bits)
    check_samples(got, ref)


def _reftex():
    import ctypes as C
    path = os.path.join(REF_DIR, "libfmvd_reftex.so")
    if not os.path.exists(path):
        pytest.skip("texture restatement not built")
    tex = C.CDLL(path)
    tex.reftex_transform.restype = C.c_int
    tex.reftex_transform.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return tex


@pytest.mark.parametrize("bits", [16, 8])
@pytest.mark.parametrize("mi", [0, 1, 2, 3])
def test_transform_vs_texture_unit(bits, mi):
    tex = _reftex()
    src = volume(bits=bits)
    frame = (24, 20, 28)
    m = np.ascontiguousarray(matrices(frame, src.shape)[mi])
    ref = np.zeros(frame, src.dtype)
    assert tex.reftex_transform(bits, src.ctypes.data, src.shape[2], src.shape[1], src.shape[0], frame[2], frame[1],
                                frame[0], m.ctypes.data, ref.ctypes.data, None, None) == 0
    got = api.transform_host(src, m, frame[2], frame[1], frame[0])
    check_vs_texture_unit(got, ref, src, m, frame, bits)


def test_transform_large_frame_vs_texture_unit():
    """A 512 x 512 frame of a rotated, z-scaled view: many TMA bricks."""
    tex = _reftex()
    rng = np.random.default_rng(5)
    src = rng.integers(0, 65535, (40, 128, 136)).astype(np.uint16)
    frame = (96, 128, 136)
    for ang in (0.0, 90.0, 180.0, 270.0):
        m = np.ascontiguousarray(synth.rotation_y_inverse(ang, frame, src.shape, 3.0, (2.0, -3.0, 1.0)))
        ref = np.zeros(frame, np.uint16)
        assert tex.reftex_transform(16, src.ctypes.data, src.shape[2], src.shape[1], src.shape[0], frame[2],
                                    frame[1], frame[0], m.ctypes.data, ref.ctypes.data, None, None) == 0
        got = api.transform_host(src, m, frame[2], frame[1], frame[0])
        check_vs_texture_unit(got, ref, src, m, frame, 16)


@pytest.mark.parametrize("bits", [16, 8])
def test_transform_float_frame_vs_oracle(bits):
    """The float frame (d_outf: the blend in sample units before
    quantisation) against the oracle's unquantised value: within float
    rounding where the 1/256 weights agree, within one weight step per axis
    elsewhere; and the sample frame written beside it is exactly the float
    frame quantised, (sample)(v / (2^bits - 1) * 2^bits + 0.5) in float."""
    import torch
    src = volume(bits=bits, shape=(30, 40, 44))
    d, h, w = src.shape
    frame = (50, 40, 44)
    pitch = api.source_pitch(bits, w)
    padded = np.zeros((d, h, pitch), src.dtype)
    padded[:, :, :w] = src
    dev = torch.from_numpy(padded.view(np.int16) if bits == 16 else padded).cuda()
    maxv = float((1 << bits) - 1)
    for m in matrices(frame, src.shape):
        out = torch.zeros(frame, dtype=torch.int16 if bits == 16 else torch.uint8, device="cuda")
        outf = torch.zeros(frame, dtype=torch.float32, device="cuda")
        api.transform_device(dev, pitch, w, h, d, m, frame[2], frame[1], 0, frame[0], out=out, out_f32=outf,
                             bits=bits)
        torch.cuda.synchronize()
        gf = outf.cpu().numpy()
        gs = out.cpu().numpy().view(np.uint16) if bits == 16 else out.cpu().numpy()
        ref = O.transform_volume(src, m, *frame, bits=bits, out_float=True) * maxv
        diff = np.abs(gf.astype(np.float64) - ref)
        sens = O.transform_weight_sensitivity(src, m, *frame, bits=bits)
        assert np.all(diff <= sens + 0.05), (diff - sens).max()
        assert (diff <= 0.05).mean() > 0.98
        q = np.floor(gf * np.float32(1.0 / maxv) * np.float32(1 << bits) + np.float32(0.5)).astype(np.int64)
        np.testing.assert_array_equal(gs.astype(np.int64), q % (1 << bits))


def test_transform_file_and_mask(tmp_path):
    src = volume()
    frame = (24, 20, 28)
    m = matrices(frame, src.shape)[1]
    outp, maskp = str(tmp_path / "t.raw"), str(tmp_path / "m.raw")
    api.transform_file(src, m, frame[2], frame[1], frame[0], outp, mask=True, border=6, zspacing=2.0, maskfile=maskp)
    got = np.fromfile(outp, np.uint16).reshape(frame)
    check_samples(got, O.transform_volume(src, m, *frame))
    mask = np.fromfile(maskp, np.float32).reshape(frame[1], frame[2])
    ref = O.transformed_mask(m, frame[0] // 2, src.shape[2], src.shape[1], src.shape[0], 2.0, frame[2], frame[1], 6.0)
    assert np.abs(mask - ref).max() < 1e-5


def test_transform_single_plane_writes_leading_plane(tmp_path):
    """For td == 1 the reference writes an unfilled slot before plane 0."""
    src = volume()
    m = matrices((1, 20, 28), src.shape)[0]
    outp = str(tmp_path / "t1.raw")
    api.transform_file(src, m, 28, 20, 1, outp)
    got = np.fromfile(outp, np.uint16).reshape(2, 20, 28)
    check_samples(got[1:], O.transform_volume(src, m, 1, 20, 28))


def test_mask_device_vs_oracle():
    import torch
    src_shape = (40, 64, 80)
    frame = (60, 64, 80)
    for ang in (0.0, 90.0):
        m = synth.rotation_y_inverse(ang, frame, src_shape, 3.0, (0.0, 0.0, 0.0))
        out = torch.zeros((frame[1], frame[2]), dtype=torch.float32, device="cuda")
        api.mask_device(out, 30, src_shape[2], src_shape[1], src_shape[0], 3.0, frame[2], frame[1], 10.0, m)
        torch.cuda.synchronize()
        ref = O.transformed_mask(m, 30, src_shape[2], src_shape[1], src_shape[0], 3.0, frame[2], frame[1], 10.0)
        assert np.abs(out.cpu().numpy() - ref).max() < 1e-5
