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

// Eight consecutive bf16 channels (16 bytes) <-> floats.
__device__ __forceinline__ void load8(const bf16 *p, float (&f)[8])
{
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float2 t = __bfloat1622float2(h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}
__device__ __forceinline__ void store8(bf16 *p, const float (&f)[8])
{
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; i++)
        h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    *reinterpret_cast<uint4 *>(p) = u;
}

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

// Grid-stride loop over n items.
#define FOR_ITEMS(i, n) \
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

// Per-plane sums in kScaleParts fixed parts (deterministic), 8 samples per load.
__global__ void plane_scale_parts_kernel(const unsigned short *views, size_t view_stride, int V, int HW, float *parts)
{
    __shared__ float red[32];
    const int n = blockIdx.y, part = blockIdx.x;
    const int chunks = HW / 8;
    const int per = (chunks + kScaleParts - 1) / kScaleParts;
    const int c0 = part * per, c1 = min(chunks, c0 + per);
    float acc = 0.f;
    for (int v = 0; v < V; v++) {
        const uint4 *p = reinterpret_cast<const uint4 *>(views + v * view_stride + (size_t)n * HW);
        for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
            const uint4 u = p[c];
            const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
                acc += (float)(w[i] & 0xFFFFu) + (float)(w[i] >> 16);
        }
    }
    const float t = block_sum(acc, red);
    if (threadIdx.x == 0)
        parts[(size_t)n * kScaleParts + part] = t;
}

// s[n] = 1 + mean over views and pixels of plane n
__global__ void plane_scale_final_kernel(const float *parts, int N, float inv_count, float *scale)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N)
        return;
    float t = 0.f;
    for (int i = 0; i < kScaleParts; i++)
        t += parts[(size_t)n * kScaleParts + i];
    scale[n] = 1.f + t * inv_count;
}

// col[n][y][x][k], k = t * (V + 1) + c: view c (c < V) or the views' mean
// (c = V), divided by s[n], at (y + dy_t, x + dx_t), zero outside; k beyond
// 9 (V + 1) zero.  A block builds kPatchPixels consecutive pixels' rows in
// shared memory (one (pixel, tap) item per thread step, loads coalesced
// along pixels), then writes them with 16-byte coalesced stores.
constexpr int kPatchPixels = 128;
__global__ void __launch_bounds__(256) input_patches_kernel(const unsigned short *views, size_t view_stride, int V,
                                                            int N, int H, int W, const float *scale, bf16 *col)
{
    __shared__ __align__(16) bf16 rows[kPatchPixels * kInputChannels];
    const size_t P = (size_t)N * H * W;
    for (size_t p0 = (size_t)blockIdx.x * kPatchPixels; p0 < P; p0 += (size_t)gridDim.x * kPatchPixels) {
        const int np = P - p0 < (size_t)kPatchPixels ? (int)(P - p0) : kPatchPixels;
        for (int i = threadIdx.x; i < kPatchPixels * kInputChannels / 8; i += blockDim.x)
            reinterpret_cast<uint4 *>(rows)[i] = make_uint4(0, 0, 0, 0);
        __syncthreads();
        for (int item = threadIdx.x; item < 9 * kPatchPixels; item += blockDim.x) {
            const int t = item / kPatchPixels, i = item % kPatchPixels;
            if (i >= np)
                continue;
            const size_t p = p0 + i;
            const int x = (int)(p % W), y = (int)((p / W) % H), n = (int)(p / ((size_t)W * H));
            const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
            if (yy < 0 || yy >= H || xx < 0 || xx >= W)
                continue;
            const float inv = 1.f / scale[n];
            const size_t q = ((size_t)n * H + yy) * W + xx;
            bf16 *r = rows + i * kInputChannels + t * (V + 1);
            float mean = 0.f;
            for (int c = 0; c < V; c++) {
                const float v = (float)views[c * view_stride + q] * inv;
                r[c] = f2b(v);
                mean += v;
            }
            r[V] = f2b(mean / (float)V);
        }
        __syncthreads();
        uint4 *dst = reinterpret_cast<uint4 *>(col + p0 * kInputChannels);
        for (int i = threadIdx.x; i < np * kInputChannels / 8; i += blockDim.x)
            dst[i] = reinterpret_cast<const uint4 *>(rows)[i];
        __syncthreads();
    }
}

// out (H/2 x W/2) = average of 2 x 2 blocks
__global__ void avgpool_kernel(const bf16 *in, bf16 *out, int N, int H, int W, int C)
{
    const int Ho = H / 2, Wo = W / 2, C8 = C / 8;
    const size_t total = (size_t)N * Ho * Wo * C8;
    FOR_ITEMS(i, total) {
        const int cc = (int)(i % C8);
        const size_t p = i / C8;
        const int x = (int)(p % Wo), y = (int)((p / Wo) % Ho), n = (int)(p / ((size_t)Wo * Ho));
        const bf16 *b = in + (((size_t)n * H + 2 * y) * W + 2 * x) * C + 8 * cc;
        float a[8], t[8];
        load8(b, a);
        load8(b + C, t);
#pragma unroll
        for (int e = 0; e < 8; e++)
            a[e] += t[e];
        load8(b + (size_t)W * C, t);
#pragma unroll
        for (int e = 0; e < 8; e++)
            a[e] += t[e];
        load8(b + (size_t)W * C + C, t);
#pragma unroll
        for (int e = 0; e < 8; e++)
            a[e] = 0.25f * (a[e] + t[e]);
        store8(out + p * C + 8 * cc, a);
    }
}

// out (2H x 2W) = nearest upsampling of in (H x W), 16 bytes per thread
__global__ void upsample_kernel(const bf16 *in, bf16 *out, int N, int H, int W, int C)
{
    const int Ho = 2 * H, Wo = 2 * W, C8 = C / 8;
    const size_t total = (size_t)N * Ho * Wo * C8;
    FOR_ITEMS(i, total) {
        const int cc = (int)(i % C8);
        const size_t p = i / C8;
        const int x = (int)(p % Wo), y = (int)((p / Wo) % Ho), n = (int)(p / ((size_t)Wo * Ho));
        reinterpret_cast<uint4 *>(out)[i] =
            *reinterpret_cast<const uint4 *>(in + (((size_t)n * H + y / 2) * W + x / 2) * C + 8 * cc);
    }
}

// Gradient at a pooled layer's input: g (H x W) = (upsampled g_pool / 4 +
// g_skip) where act > 0, else 0.
__global__ void pool_grad_kernel(const bf16 *g_pool, const bf16 *g_skip, const bf16 *act, bf16 *g, int N, int H,
                                 int W, int C)
{
    const int Hp = H / 2, Wp = W / 2, C8 = C / 8;
    const size_t total = (size_t)N * H * W * C8;
    FOR_ITEMS(i, total) {
        const int cc = (int)(i % C8);
        const size_t p = i / C8;
        const int x = (int)(p % W), y = (int)((p / W) % H), n = (int)(p / ((size_t)W * H));
        float v[8], a[8], k[8];
        load8(g_pool + (((size_t)n * Hp + y / 2) * Wp + x / 2) * C + 8 * cc, v);
        load8(act + p * C + 8 * cc, a);
        if (g_skip)
            load8(g_skip + p * C + 8 * cc, k);
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const float t = 0.25f * v[e] + (g_skip ? k[e] : 0.f);
            v[e] = a[e] > 0.f ? t : 0.f;
        }
        store8(g + p * C + 8 * cc, v);
    }
}

// Gradient at an upsampled layer's input: g (H x W) = sum of the 2 x 2
// block of g_up (2H x 2W) where act > 0, else 0.
__global__ void upsample_grad_kernel(const bf16 *g_up, const bf16 *act, bf16 *g, int N, int H, int W, int C)
{
    const int Wu = 2 * W, C8 = C / 8;
    const size_t total = (size_t)N * H * W * C8;
    FOR_ITEMS(i, total) {
        const int cc = (int)(i % C8);
        const size_t p = i / C8;
        const int x = (int)(p % W), y = (int)((p / W) % H), n = (int)(p / ((size_t)W * H));
        const bf16 *b = g_up + (((size_t)n * 2 * H + 2 * y) * Wu + 2 * x) * C + 8 * cc;
        float s[8], t[8], a[8];
        load8(b, s);
        load8(b + C, t);
#pragma unroll
        for (int e = 0; e < 8; e++)
            s[e] += t[e];
        load8(b + (size_t)Wu * C, t);
#pragma unroll
        for (int e = 0; e < 8; e++)
            s[e] += t[e];
        load8(b + (size_t)Wu * C + C, t);
        load8(act + p * C + 8 * cc, a);
#pragma unroll
        for (int e = 0; e < 8; e++)
            s[e] = a[e] > 0.f ? s[e] + t[e] : 0.f;
        store8(g + p * C + 8 * cc, s);
    }
}

// db[c] += sum over pixels of g[p][c]: thread (row r, chunk cc) sums 8
// channels over pixels r, r + rows, ...; block partials through shared memory.
__global__ void bias_grad_kernel(const bf16 *g, size_t P, int C, float *db)
{
    __shared__ float sdb[256];
    const int C8 = C / 8;
    const int rows = blockDim.x / C8;
    const int cc = threadIdx.x % C8, r = threadIdx.x / C8;
    for (int i = threadIdx.x; i < C; i += blockDim.x)
        sdb[i] = 0.f;
    __syncthreads();
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (r < rows) {
        for (size_t p = blockIdx.x * (size_t)rows + r; p < P; p += (size_t)gridDim.x * rows) {
            float v[8];
            load8(g + p * C + 8 * cc, v);
#pragma unroll
            for (int e = 0; e < 8; e++)
                acc[e] += v[e];
        }
#pragma unroll
        for (int e = 0; e < 8; e++)
            atomicAdd(&sdb[8 * cc + e], acc[e]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < C; i += blockDim.x)
        atomicAdd(db + i, sdb[i]);
}

// y[p] = sum_c act[p][c] w[c] + b (normalised units); optional outputs:
// the estimate y * s[n], and with a target the L1 loss and its gradient.
__global__ void output_kernel(const bf16 *act, const float *w, const float *b, int C, int N, int HW,
                              const float *scale, float *estimate, const float *target, float *gy, float inv_count,
                              float *loss)
{
    __shared__ float red[32];
    __shared__ float sw[kMaxOutChannels];
    for (int i = threadIdx.x; i < C; i += blockDim.x)
        sw[i] = w[i];
    __syncthreads();
    const size_t total = (size_t)N * HW;
    const float b0 = b[0];
    float lsum = 0.f;
    FOR_ITEMS(p, total) {
        float y = b0;
        for (int c0 = 0; c0 < C; c0 += 8) {
            float a[8];
            load8(act + p * C + c0, a);
#pragma unroll
            for (int e = 0; e < 8; e++)
                y += a[e] * sw[c0 + e];
        }
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
    __shared__ float sw[kMaxOutChannels];
    for (int i = threadIdx.x; i <= C; i += blockDim.x) {
        sdw[i] = 0.f;
        if (i < C)
            sw[i] = w[i];
    }
    __syncthreads();
    float pdw[kMaxOutChannels];
#pragma unroll
    for (int c = 0; c < kMaxOutChannels; c++)
        pdw[c] = 0.f;
    float pdb = 0.f;
    FOR_ITEMS(p, P) {
        const float g = gy[p];
        pdb += g;
#pragma unroll
        for (int c0 = 0; c0 < kMaxOutChannels; c0 += 8) {
            if (c0 >= C)
                break;
            float a[8], o[8];
            load8(act + p * C + c0, a);
#pragma unroll
            for (int e = 0; e < 8; e++) {
                pdw[c0 + e] += g * a[e];
                o[e] = a[e] > 0.f ? g * sw[c0 + e] : 0.f;
            }
            store8(g_act + p * C + c0, o);
        }
    }
#pragma unroll
    for (int c = 0; c < kMaxOutChannels; c++)
        if (c < C)
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
                            float b2, float eps, const float *gscale)
{
    const float sc = gscale ? *gscale : 1.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float g = grad[i] * sc;
        const float mi = b1 * m[i] + (1.f - b1) * g;
        const float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        param[i] -= lr_t * mi / (sqrtf(vi) + eps);
    }
}

// Squared L2 norm of the gradient, added into *out (zeroed by the caller).
__global__ void grad_norm2_kernel(const float *g, size_t n, float *out)
{
    float acc = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        acc = fmaf(g[i], g[i], acc);
    for (int o = 16; o; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(out, acc);
}

// Adaptive clipping of one step: state[0] = the step's squared gradient
// norm, state[1] = running mean of the (clipped) norms of earlier steps (0
// before the first), state[2] = the factor Adam applies to this step's
// gradient: limit / norm where the norm exceeds limit = factor x the running
// mean, 0 for a non-finite norm (the step is skipped), else 1.
__global__ void clip_scale_kernel(float *state, float factor)
{
    const float norm = sqrtf(state[0]);
    if (!isfinite(norm)) {
        state[2] = 0.f;
        return;
    }
    const float mean = state[1] > 0.f ? state[1] : norm;
    const float limit = factor * mean;
    state[2] = norm > limit && norm > 0.f ? limit / norm : 1.f;
    state[1] = 0.95f * mean + 0.05f * fminf(norm, limit);
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
    float *parts = scale + N;
    plane_scale_parts_kernel<<<dim3(kScaleParts, N), 256, 0, s>>>(views, view_stride, V, HW, parts);
    plane_scale_final_kernel<<<(N + 127) / 128, 128, 0, s>>>(parts, N, 1.f / (float)((size_t)V * HW), scale);
    rl_count_launch(2);
    return FMVD_CHECK(cudaGetLastError());
}

bool input_patches(const unsigned short *views, size_t view_stride, int V, int N, int H, int W, const float *scale,
                   bf16 *col, cudaStream_t s)
{
    const size_t groups = ((size_t)N * H * W + kPatchPixels - 1) / kPatchPixels;
    input_patches_kernel<<<(int)(groups < 148 * 8 ? groups : 148 * 8), 256, 0, s>>>(views, view_stride, V, N, H, W,
                                                                                   scale, col);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool avgpool(const bf16 *in, bf16 *out, int N, int H, int W, int C, cudaStream_t s)
{
    avgpool_kernel<<<grid_for((size_t)N * H * W * C / 32), 256, 0, s>>>(in, out, N, H, W, C);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool upsample(const bf16 *in, bf16 *out, int N, int H, int W, int C, cudaStream_t s)
{
    upsample_kernel<<<grid_for((size_t)N * H * W * C / 2), 256, 0, s>>>(in, out, N, H, W, C);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool pool_grad(const bf16 *g_pool, const bf16 *g_skip, const bf16 *act, bf16 *g, int N, int H, int W, int C,
               cudaStream_t s)
{
    pool_grad_kernel<<<grid_for((size_t)N * H * W * C / 8), 256, 0, s>>>(g_pool, g_skip, act, g, N, H, W, C);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool upsample_grad(const bf16 *g_up, const bf16 *act, bf16 *g, int N, int H, int W, int C, cudaStream_t s)
{
    upsample_grad_kernel<<<grid_for((size_t)N * H * W * C / 8), 256, 0, s>>>(g_up, act, g, N, H, W, C);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool bias_grad(const bf16 *g, size_t P, int C, float *db, cudaStream_t s)
{
    // 256 threads: C / 8 channel chunks by 256 / (C / 8) pixel rows
    const size_t rows = 256 / (C / 8);
    const size_t need = (P + rows - 1) / rows;
    bias_grad_kernel<<<(int)(need < 148 * 8 ? need : 148 * 8), 256, 0, s>>>(g, P, C, db);
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
          cudaStream_t s, float *clip_state, float clip_factor)
{
    if (clip_state) {
        if (!FMVD_CHECK(cudaMemsetAsync(clip_state, 0, sizeof(float), s)))
            return false;
        grad_norm2_kernel<<<grid_for(n), 256, 0, s>>>(grad, n, clip_state);
        clip_scale_kernel<<<1, 1, 0, s>>>(clip_state, clip_factor);
        rl_count_launch(2);
    }
    adam_kernel<<<grid_for(n), 256, 0, s>>>(param, grad, m, v, n, lr_t, b1, b2, eps,
                                            clip_state ? clip_state + 2 : nullptr);
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
