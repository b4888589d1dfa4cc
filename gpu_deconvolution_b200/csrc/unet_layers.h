// Layer kernels of the warm-start network (unet_layers.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>

namespace fmvd {
namespace unet {

constexpr int kInputChannels = 64;   // first-layer patch channels: 9 taps x (views + mean), zero padded
constexpr int kMaxOutChannels = 64;  // channels feeding the 1x1 output layer
constexpr int kScaleParts = 64;      // fixed parts of the per-plane scale reduction

// Channel counts of the layer kernels are multiples of 8 (16-byte vectors),
// at most 256.  plane_scale: scale holds N * (kScaleParts + 1) floats, the
// first N receive the scales.

bool plane_scale(const unsigned short *views, size_t view_stride, int V, int N, int HW, float *scale, cudaStream_t s);
bool input_patches(const unsigned short *views, size_t view_stride, int V, int N, int H, int W, const float *scale,
                   __nv_bfloat16 *col, cudaStream_t s);
bool avgpool(const __nv_bfloat16 *in, __nv_bfloat16 *out, int N, int H, int W, int C, cudaStream_t s);
bool upsample(const __nv_bfloat16 *in, __nv_bfloat16 *out, int N, int H, int W, int C, cudaStream_t s);
bool pool_grad(const __nv_bfloat16 *g_pool, const __nv_bfloat16 *g_skip, const __nv_bfloat16 *act, __nv_bfloat16 *g,
               int N, int H, int W, int C, cudaStream_t s);
bool upsample_grad(const __nv_bfloat16 *g_up, const __nv_bfloat16 *act, __nv_bfloat16 *g, int N, int H, int W, int C,
                   cudaStream_t s);
bool bias_grad(const __nv_bfloat16 *g, size_t P, int C, float *db, cudaStream_t s);
bool output_layer(const __nv_bfloat16 *act, const float *w, const float *b, int C, int N, int HW, const float *scale,
                  float *estimate, const float *target, float *gy, float *loss, cudaStream_t s);
bool output_grad(const __nv_bfloat16 *act, const float *w, int C, size_t P, const float *gy, __nv_bfloat16 *g_act,
                 float *dw, float *db, cudaStream_t s);
// One Adam step.  With clip_state (3 floats on the device, zeroed before the
// first step) the gradient is first clipped adaptively: scaled down to
// clip_factor x the running mean of earlier steps' norms where its L2 norm
// exceeds that, and the step skipped where the norm is not finite.
bool adam(float *param, const float *grad, float *m, float *v, size_t n, float lr_t, float b1, float b2, float eps,
          cudaStream_t s, float *clip_state = nullptr, float clip_factor = 2.f);
bool weight_copies(const float *w, int cout, int taps, int cin, __nv_bfloat16 *wf, __nv_bfloat16 *wt, cudaStream_t s);

} // namespace unet
} // namespace fmvd
