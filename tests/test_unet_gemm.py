"""Tensor-core convolution GEMMs of the warm-start network
(fmvd_b200_conv_bf16, fmvd_b200_conv_wgrad_bf16) against the FP64 oracle.

Inputs are bf16 values, so the oracle sees exactly what the tensor cores
multiply; the only difference is the FP32 accumulation order, hence the
tight tolerances.  CPU tests pin the oracle's own adjoint identities."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import unet_oracle as U


def test_oracle_adjoints():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(2, 6, 5, 4))
    w = rng.normal(size=(3, 9, 4))
    g = rng.normal(size=(2, 6, 5, 3))
    y = U.conv(x, w)
    # data gradient = convolution with the flipped, transposed kernel
    dx = U.conv(g, U.conv_dgrad_weights(w))
    assert np.isclose(np.sum(y * g), np.sum(x * dx))
    # weight gradient
    dw = U.conv_wgrad(g, x, 9)
    assert np.isclose(np.sum(y * g), np.sum(w * dw))


def test_bf16_round():
    a = np.array([1.0, 1.00390625, 1.0078125, -3.14159, 65504.0], np.float32)
    r = U.bf16_round(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125  # ties to even
    assert abs(r[3] + 3.140625) < 1e-6


def _bf(torch, shape, g, scale=1.0):
    return (torch.randn(shape, generator=g, device="cuda") * scale).to(torch.bfloat16)


def _np(t):
    return t.float().cpu().numpy()


CONV_CASES = [
    # N, H, W, cin, cout, taps
    (2, 16, 16, 32, 32, 9),
    (1, 8, 32, 64, 16, 9),
    (2, 16, 16, 64, 64, 1),
    (1, 16, 8, 128, 256, 9),
    (1, 8, 128, 32, 128, 9),
    (1, 4, 256, 64, 512, 9),
]


@pytest.mark.gpu
@pytest.mark.parametrize("N,H,W,cin,cout,taps", CONV_CASES)
def test_conv_forward_matches_oracle(N, H, W, cin, cout, taps):
    import torch
    from gpu_deconvolution_b200 import native
    lib = native.load()
    g = torch.Generator(device="cuda").manual_seed(cin * 7 + cout)
    x = _bf(torch, (N, H, W, cin), g)
    w = _bf(torch, (cout, taps, cin), g, 0.1)
    bias = torch.randn(cout, generator=g, device="cuda")
    add = _bf(torch, (N, H, W, cout), g)
    mask = _bf(torch, (N, H, W, cout), g)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for use_extra in (False, True):
        out = torch.zeros((N, H, W, cout), dtype=torch.bfloat16, device="cuda")
        outf = torch.zeros((N, H, W, cout), dtype=torch.float32, device="cuda")
        native.clear_errors()
        r = lib.fmvd_b200_conv_bf16(x.data_ptr(), w.data_ptr(), N, H, W, cin, cout, taps, out.data_ptr(),
                                    outf.data_ptr(), bias.data_ptr() if use_extra else None,
                                    add.data_ptr() if use_extra else None, mask.data_ptr() if use_extra else None,
                                    int(use_extra), status.data_ptr(), None)
        native.check("fmvd_b200_conv_bf16")
        assert r == 0
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        if use_extra:
            ref = U.conv(_np(x), _np(w), _np(bias), _np(add), True, _np(mask))
        else:
            ref = U.conv(_np(x), _np(w))
        assert rel_l2(_np(outf), ref) < 1e-5
        np.testing.assert_array_equal(_np(out), U.bf16_round(_np(outf)))


WGRAD_CASES = [
    # N, H, W, cin, cout, taps
    (2, 16, 16, 32, 32, 9),
    (1, 16, 64, 64, 32, 9),
    (2, 8, 8, 32, 64, 1),
    (1, 16, 16, 128, 128, 9),
    (1, 8, 64, 256, 256, 9),
    (1, 8, 128, 64, 128, 1),
]


@pytest.mark.gpu
@pytest.mark.parametrize("N,H,W,cin,cout,taps", WGRAD_CASES)
def test_conv_wgrad_matches_oracle(N, H, W, cin, cout, taps):
    import torch
    from gpu_deconvolution_b200 import native
    lib = native.load()
    g = torch.Generator(device="cuda").manual_seed(cin * 11 + cout)
    grad = _bf(torch, (N, H, W, cout), g)
    x = _bf(torch, (N, H, W, cin), g)
    dw = torch.zeros((cout, taps, cin), dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    native.clear_errors()
    r = lib.fmvd_b200_conv_wgrad_bf16(grad.data_ptr(), x.data_ptr(), N, H, W, cin, cout, taps, dw.data_ptr(),
                                      status.data_ptr(), None)
    native.check("fmvd_b200_conv_wgrad_bf16")
    assert r == 0
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ref = U.conv_wgrad(_np(grad), _np(x), taps)
    assert rel_l2(dw.cpu().numpy(), ref) < 1e-5


@pytest.mark.gpu
def test_conv_dgrad_through_flipped_weights():
    """The data gradient is the forward GEMM on the flipped, transposed kernel."""
    import torch
    from gpu_deconvolution_b200 import native
    lib = native.load()
    N, H, W, cin, cout = 2, 16, 16, 32, 64
    g = torch.Generator(device="cuda").manual_seed(5)
    grad = _bf(torch, (N, H, W, cout), g)
    w = _bf(torch, (cout, 9, cin), g, 0.1)
    wt = torch.from_numpy(U.conv_dgrad_weights(_np(w))).cuda().to(torch.bfloat16).contiguous()
    outf = torch.zeros((N, H, W, cin), dtype=torch.float32, device="cuda")
    r = lib.fmvd_b200_conv_bf16(grad.data_ptr(), wt.data_ptr(), N, H, W, cout, cin, 9, None, outf.data_ptr(),
                                None, None, None, 0, None, None)
    assert r == 0
    torch.cuda.synchronize()
    ref = U.conv(_np(grad), U.conv_dgrad_weights(_np(w)))
    assert rel_l2(_np(outf), ref) < 1e-5
