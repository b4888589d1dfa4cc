// Warm-start network: tensor-core convolution GEMMs and the layer kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>

namespace fmvd {
namespace unet {

// Kernel arguments of the convolution GEMM (see unet_gemm.cu).
struct GemmArgs {
    int N, H, W;          // images and image size of the pixel grid
    int bw, bh;           // pixel box of one tile (mode 0) or K block (mode 1)
    int taps;             // 9 (3 x 3) or 1
    int cin, cout;        // channels of the input / output of the convolution
    int kchunk;           // mode 1: pixel K blocks per CTA
    __nv_bfloat16 *out;   // mode 0 outputs
    int out_ld, out_coff;
    float *out_f32;
    int outf_ld;
    const float *bias;
    const __nv_bfloat16 *add;
    int add_ld;
    const __nv_bfloat16 *mask;
    int mask_ld;
    int relu;
    float *dw;            // mode 1 output, [cout][taps][cin], accumulated
    int *status;          // set to 1 when a wait timed out
};

// out[n][y][x][co] = act(sum_{t, ci} in[n][y + dy_t][x + dx_t][ci] * weight[co][t][ci]
//                        + bias[co] + add[n][y][x][co]), zero where mask <= 0.
// cin a multiple of 32, cout of 16 (<= 256 or a multiple of 256), W a
// multiple of 8 that divides or is divided by 128.
struct ConvDesc {
    const __nv_bfloat16 *in;
    const __nv_bfloat16 *weight;
    int N, H, W, cin, cout, taps;
    __nv_bfloat16 *out;
    int out_ld, out_coff;  // 0 -> cout, 0
    float *out_f32;
    int outf_ld;
    const float *bias;
    const __nv_bfloat16 *add;
    int add_ld;
    const __nv_bfloat16 *mask;
    int mask_ld;
    int relu;
    int *status;
};

// dw[co][t][ci] += sum_{n, y, x} grad[n][y][x][co] * in[n][y + dy_t][x + dx_t][ci]
struct WgradDesc {
    const __nv_bfloat16 *grad;
    const __nv_bfloat16 *in;
    int N, H, W, cin, cout, taps;
    float *dw;
    int *status;
};

bool conv_forward(const ConvDesc &c, cudaStream_t s);
bool conv_wgrad(const WgradDesc &c, cudaStream_t s);

} // namespace unet
} // namespace fmvd
