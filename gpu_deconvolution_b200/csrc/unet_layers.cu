// Element-wise and reduction kernels of the warm-start network (BF16 NHWC
// activations, FP32 arithmetic): input normalisation and 3x3 patch
// extraction of the first layer, 2x2 average pooling / nearest upsampling
// and their gradients, bias gradients, the 1x1 output layer with the L1 loss,
// and the Adam update that also writes the bf16 weights of the forward and
// data-gradient GEMMs.
#include "fmvd_internal.h"
#include "unet_layers.h"

#include <cuda_bf16.h>

namespace fmvd {
namespace unet {

using bf16 = __nv_bfloat16;

namespace {

__device__ __forceinline__ float b2f(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ bf16 f2b(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ float block_sum(float v, float *red)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0)
        red[warp] = v;
    __syncthreads();
    float t = 0.f;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++)
            t += red[w];
    return t;
}

// s[n] = 1 + mean over views and pixels of plane n
__global__ void plane_scale_kernel(const unsigned short *views, size_t view_stride, int V, int HW, float *scale)
{
    __shared__ float red[32];
    const int n = blockIdx.x;
    float acc = 0.f;
    for (int v = 0; v < V; v++) {
        const unsigned short *p = views + v * view_stride + (size_t)n * HW;
        for (int i = threadIdx.x; i < HW; i += blockDim.x)
            acc += (float)p[i];
    }
    const float t = block_sum(acc, red);
    if (threadIdx.x == 0)
        scale[n] = 1.f + t / (float)(V * HW);
}

// col[n][y][x][t * (V + 1) + c]: view c (c < V) or the views' mean (c = V),
// divided by s[n], at (y + dy_t, x + dx_t), zero outside; channels beyond
// 9 (V + 1) are zero.
__global__ void input_patches_kernel(const unsigned short *views, size_t view_stride, int V, int N, int H, int W,
                                     const float *scale, bf16 *col)
{
    const size_t total = (size_t)N * H * W;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % W), y = (int)((p / W) % H), n = (int)(p / ((size_t)W * H));
        const float inv = 1.f / scale[n];
        __align__(16) bf16 out[kInputChannels];
#pragma unroll
        for (int k = 0; k < kInputChannels; k++)
            out[k] = f2b(0.f);
        for (int t = 0; t < 9; t++) {
            const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
            if (yy < 0 || yy >= H || xx < 0 || xx >= W)
                continue;
            float mean = 0.f;
            for (int c = 0; c < V; c++) {
                const float v = (float)views[c * view_stride + ((size_t)n * H + yy) * W + xx] * inv;
                out[t * (V + 1) + c] = f2b(v);
                mean += v;
            }
            out[t * (V + 1) + V] = f2b(mean / (float)V);
        }
        uint4 *dst = reinterpret_cast<uint4 *>(col + p * kInputChannels);
#pragma unroll
        for (int i = 0; i < kInputChannels / 8; i++)
            dst[i] = reinterpret_cast<const uint4 *>(out)[i];
    }
}

// out (H/2 x W/2) = average of 2 x 2 blocks
__global__ void avgpool_kernel(const bf16 *in, bf16 *out, int N, int H, int W, int C)
{
    const int Ho = H / 2, Wo = W / 2;
    const size_t total = (size_t)N * Ho * Wo * C;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const size_t p = i / C;
        const int x = (int)(p % Wo), y = (int)((p / Wo) % Ho), n = (int)(p / ((size_t)Wo * Ho));
        const size_t b = (((size_t)n * H + 2 * y) * W + 2 * x) * C + c;
        const float s = b2f(in[b]) + b2f(in[b + C]) + b2f(in[b + (size_t)W * C]) + b2f(in[b + (size_t)W * C + C]);
        out[i] = f2b(0.25f * s);
    }
}

// out (2H x 2W) = nearest upsampling of in (H x W)
__global__ void upsample_kernel(const bf16 *in, bf16 *out, int N, int H, int W, int C)
{
    const int Ho = 2 * H, Wo = 2 * W;
    const size_t total = (size_t)N * Ho * Wo * C;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const size_t p = i / C;
        const int x = (int)(p % Wo), y = (int)((p / Wo) % Ho), n = (int)(p / ((size_t)Wo * Ho));
        out[i] = in[(((size_t)n * H + y / 2) * W + x / 2) * C + c];
    }
}

// Gradient at a pooled layer's input: g (H x W) = (upsampled g_pool / 4 +
// g_skip) where act > 0, else 0.
__global__ void pool_grad_kernel(const bf16 *g_pool, const bf16 *g_skip, const bf16 *act, bf16 *g, int N, int H,
                                 int W, int C)
{
    const size_t total = (size_t)N * H * W * C;
    const int Hp = H / 2, Wp = W / 2;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const size_t p = i / C;
        const int x = (int)(p % W), y = (int)((p / W) % H), n = (int)(p / ((size_t)W * H));
        float v = 0.25f * b2f(g_pool[(((size_t)n * Hp + y / 2) * Wp + x / 2) * C + c]);
        if (g_skip)
            v += b2f(g_skip[i]);
        g[i] = f2b(b2f(act[i]) > 0.f ? v : 0.f);
    }
}

// Gradient at an upsampled layer's input: g (H x W) = sum of the 2 x 2
// block of g_up (2H x 2W) where act > 0, else 0.
__global__ void upsample_grad_kernel(const bf16 *g_up, const bf16 *act, bf16 *g, int N, int H, int W, int C)
{
    const size_t total = (size_t)N * H * W * C;
    const int Wu = 2 * W;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const size_t p = i / C;
        const int x = (int)(p % W), y = (int)((p / W) % H), n = (int)(p / ((size_t)W * H));
        const size_t b = (((size_t)n * 2 * H + 2 * y) * Wu + 2 * x) * C + c;
        const float s = b2f(g_up[b]) + b2f(g_up[b + C]) + b2f(g_up[b + (size_t)Wu * C]) +
                        b2f(g_up[b + (size_t)Wu * C + C]);
        g[i] = f2b(b2f(act[i]) > 0.f ? s : 0.f);
    }
}

// db[c] += sum over pixels of g[p][c]; one thread per channel per block row
__global__ void bias_grad_kernel(const bf16 *g, size_t P, int C, float *db)
{
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;
    const int l = threadIdx.x / C;
    float acc = 0.f;
    for (size_t p = blockIdx.x * (size_t)lanes + l; p < P; p += (size_t)gridDim.x * lanes)
        acc += b2f(g[p * C + c]);
    atomicAdd(db + c, acc);
}

// y[p] = sum_c act[p][c] w[c] + b (normalised units); optional outputs:
// the estimate y * s[n], and with a target the L1 loss and its gradient.
__global__ void output_kernel(const bf16 *act, const float *w, const float *b, int C, int N, int HW,
                              const float *scale, float *estimate, const float *target, float *gy, float inv_count,
                              float *loss)
{
    __shared__ float red[32];
    const size_t total = (size_t)N * HW;
    float lsum = 0.f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        float y = b[0];
        for (int c = 0; c < C; c++)
            y += b2f(act[p * C + c]) * w[c];
        const int n = (int)(p / HW);
        if (estimate)
            estimate[p] = y * scale[n];
        if (target) {
            const float d = y - target[p] / scale[n];
            lsum += fabsf(d);
            gy[p] = (d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f)) * inv_count;
        }
    }
    if (target && loss) {
        const float t = block_sum(lsum, red);
        if (threadIdx.x == 0)
            atomicAdd(loss, t * inv_count);
    }
}

// g_act[p][c] = gy[p] w[c] where act > 0; dw[c] += sum_p gy[p] act[p][c]; db += sum_p gy[p]
__global__ void output_grad_kernel(const bf16 *act, const float *w, int C, size_t P, const float *gy, bf16 *g_act,
                                   float *dw, float *db)
{
    __shared__ float sdw[kMaxOutChannels + 1];
    for (int i = threadIdx.x; i <= C; i += blockDim.x)
        sdw[i] = 0.f;
    __syncthreads();
    float pdw[kMaxOutChannels];
    for (int c = 0; c < C; c++)
        pdw[c] = 0.f;
    float pdb = 0.f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < P; p += (size_t)gridDim.x * blockDim.x) {
        const float g = gy[p];
        pdb += g;
        for (int c = 0; c < C; c++) {
            const float a = b2f(act[p * C + c]);
            pdw[c] += g * a;
            g_act[p * C + c] = f2b(a > 0.f ? g * w[c] : 0.f);
        }
    }
    for (int c = 0; c < C; c++)
        atomicAdd(&sdw[c], pdw[c]);
    atomicAdd(&sdw[C], pdb);
    __syncthreads();
    for (int i = threadIdx.x; i < C; i += blockDim.x)
        atomicAdd(dw + i, sdw[i]);
    if (threadIdx.x == 0)
        atomicAdd(db, sdw[C]);
}

// Adam on the FP32 master parameters (bias-corrected step size lr_t).
__global__ void adam_kernel(float *param, const float *grad, float *m, float *v, size_t n, float lr_t, float b1,
                            float b2, float eps)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float g = grad[i];
        const float mi = b1 * m[i] + (1.f - b1) * g;
        const float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        param[i] -= lr_t * mi / (sqrtf(vi) + eps);
    }
}

// bf16 forward weights w[co][t][ci] and data-gradient weights
// wt[ci][taps - 1 - t][co] from the FP32 master copy.
__global__ void weight_copies_kernel(const float *w, int cout, int taps, int cin, bf16 *wf, bf16 *wt)
{
    const int total = cout * taps * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int ci = i % cin, t = (i / cin) % taps, co = i / (cin * taps);
        const bf16 h = f2b(w[i]);
        wf[i] = h;
        if (wt)
            wt[((size_t)ci * taps + (taps - 1 - t)) * cout + co] = h;
    }
}

int grid_for(size_t n, int threads = 256)
{
    size_t b = (n + threads - 1) / threads;
    return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

} // namespace

bool plane_scale(const unsigned short *views, size_t view_stride, int V, int N, int HW, float *scale, cudaStream_t s)
{
    plane_scale_kernel<<<N, 512, 0, s>>>(views, view_stride, V, HW, scale);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool input_patches(const unsigned short *views, size_t view_stride, int V, int N, int H, int W, const float *scale,
                   bf16 *col, cudaStream_t s)
{
    input_patches_kernel<<<grid_for((size_t)N * H * W), 256, 0, s>>>(views, view_stride, V, N, H, W, scale, col);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool avgpool(const bf16 *in, bf16 *out, int N, int H, int W, int C, cudaStream_t s)
{
    avgpool_kernel<<<grid_for((size_t)N * H * W * C / 4), 256, 0, s>>>(in, out, N, H, W, C);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool upsample(const bf16 *in, bf16 *out, int N, int H, int W, int C, cudaStream_t s)
{
    upsample_kernel<<<grid_for((size_t)N * H * W * C * 4), 256, 0, s>>>(in, out, N, H, W, C);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool pool_grad(const bf16 *g_pool, const bf16 *g_skip, const bf16 *act, bf16 *g, int N, int H, int W, int C,
               cudaStream_t s)
{
    pool_grad_kernel<<<grid_for((size_t)N * H * W * C), 256, 0, s>>>(g_pool, g_skip, act, g, N, H, W, C);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool upsample_grad(const bf16 *g_up, const bf16 *act, bf16 *g, int N, int H, int W, int C, cudaStream_t s)
{
    upsample_grad_kernel<<<grid_for((size_t)N * H * W * C), 256, 0, s>>>(g_up, act, g, N, H, W, C);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool bias_grad(const bf16 *g, size_t P, int C, float *db, cudaStream_t s)
{
    const int threads = C >= 256 ? C : (256 / C) * C;
    bias_grad_kernel<<<grid_for(P * C / 16, threads), threads, 0, s>>>(g, P, C, db);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool output_layer(const bf16 *act, const float *w, const float *b, int C, int N, int HW, const float *scale,
                  float *estimate, const float *target, float *gy, float *loss, cudaStream_t s)
{
    const float inv = 1.f / (float)((size_t)N * HW);
    output_kernel<<<grid_for((size_t)N * HW), 256, 0, s>>>(act, w, b, C, N, HW, scale, estimate, target, gy, inv,
                                                           loss);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool output_grad(const bf16 *act, const float *w, int C, size_t P, const float *gy, bf16 *g_act, float *dw,
                 float *db, cudaStream_t s)
{
    output_grad_kernel<<<grid_for(P), 256, 0, s>>>(act, w, C, P, gy, g_act, dw, db);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool adam(float *param, const float *grad, float *m, float *v, size_t n, float lr_t, float b1, float b2, float eps,
          cudaStream_t s)
{
    adam_kernel<<<grid_for(n), 256, 0, s>>>(param, grad, m, v, n, lr_t, b1, b2, eps);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool weight_copies(const float *w, int cout, int taps, int cin, bf16 *wf, bf16 *wt, cudaStream_t s)
{
    weight_copies_kernel<<<grid_for((size_t)cout * taps * cin), 256, 0, s>>>(w, cout, taps, cin, wf, wt);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

} // namespace unet
} // namespace fmvd
