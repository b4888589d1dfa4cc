// C entry points of the warm-start network's tensor-core convolutions.
#include "fmvd_b200.h"
#include "fmvd_internal.h"
#include "unet.h"

extern "C" {

int fmvd_b200_conv_bf16(const void *d_in, const void *d_weight, int N, int H, int W, int cin, int cout, int taps,
                        void *d_out, float *d_out_f32, const float *d_bias, const void *d_add, const void *d_mask,
                        int relu, int *d_status, void *stream)
{
    if (!d_in || !d_weight || N < 1 || H < 1 || W < 1 || (!d_out && !d_out_f32)) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_conv_bf16");
        return 1;
    }
    fmvd::unet::ConvDesc c{};
    c.in = (const __nv_bfloat16 *)d_in;
    c.weight = (const __nv_bfloat16 *)d_weight;
    c.N = N;
    c.H = H;
    c.W = W;
    c.cin = cin;
    c.cout = cout;
    c.taps = taps;
    c.out = (__nv_bfloat16 *)d_out;
    c.out_f32 = d_out_f32;
    c.bias = d_bias;
    c.add = (const __nv_bfloat16 *)d_add;
    c.mask = (const __nv_bfloat16 *)d_mask;
    c.relu = relu;
    c.status = d_status;
    return fmvd::unet::conv_forward(c, (cudaStream_t)stream) ? 0 : 1;
}

int fmvd_b200_conv_wgrad_bf16(const void *d_grad, const void *d_in, int N, int H, int W, int cin, int cout, int taps,
                              float *d_dw, int *d_status, void *stream)
{
    if (!d_grad || !d_in || !d_dw || N < 1 || H < 1 || W < 1) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_conv_wgrad_bf16");
        return 1;
    }
    fmvd::unet::WgradDesc c{};
    c.grad = (const __nv_bfloat16 *)d_grad;
    c.in = (const __nv_bfloat16 *)d_in;
    c.N = N;
    c.H = H;
    c.W = W;
    c.cin = cin;
    c.cout = cout;
    c.taps = taps;
    c.dw = d_dw;
    c.status = d_status;
    return fmvd::unet::conv_wgrad(c, (cudaStream_t)stream) ? 0 : 1;
}

} // extern "C"
