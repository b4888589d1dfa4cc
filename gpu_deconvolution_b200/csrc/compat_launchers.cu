// The reference's exported element-wise launchers (fmvd_deconvolve_cuda.cuh,
// fmvd_deconvolve_cuda.impl.cuh), kept for callers that use them directly.
// Grid-stride kernels over the whole plane; semantics per launcher are listed
// in include/fmvd_deconvolve_cuda.h.
#include "fmvd_deconvolve_cuda.h"
#include "fmvd_internal.h"

namespace {

__device__ __forceinline__ int clamp_src(int i, int n, int border)
{
    return i < n ? i : (i < n + border ? n - 1 : 0);
}

int grid_for(size_t n)
{
    size_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

#define GRID_STRIDE(i, n) for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

__global__ void k_pad_kernel(float *dst, const float *src, int fftH, int fftW, int kH, int kW)
{
    GRID_STRIDE(i, (size_t)kH * kW)
    {
        const int y = (int)(i / kW), x = (int)(i % kW);
        int ky = y - kH / 2, kx = x - kW / 2;
        if (ky < 0) ky += fftH;
        if (kx < 0) kx += fftW;
        dst[(size_t)ky * fftW + kx] = src[i];
    }
}

__global__ void k_pad_weights(float *pw, float *sums, const float *w, int fftH, int fftW, int dataH, int dataW, int by,
                              int bx)
{
    GRID_STRIDE(i, (size_t)fftH * fftW)
    {
        const int y = (int)(i / fftW), x = (int)(i % fftW);
        const float v = w[(size_t)clamp_src(y, dataH, by) * dataW + clamp_src(x, dataW, bx)];
        pw[i] = v;
        sums[i] += v;
    }
}

__global__ void k_normalize_weights(float *pw, const float *sums, size_t n)
{
    GRID_STRIDE(i, n)
    {
        const float s = sums[i];
        if (s > 0)
            pw[i] /= s;
    }
}

template <typename T>
__global__ void k_pad_clamp(T *dst, const T *src, int fftH, int fftW, int dataH, int dataW, int by, int bx)
{
    GRID_STRIDE(i, (size_t)fftH * fftW)
    {
        const int y = (int)(i / fftW), x = (int)(i % fftW);
        dst[i] = src[(size_t)clamp_src(y, dataH, by) * dataW + clamp_src(x, dataW, bx)];
    }
}

template <typename S>
__global__ void k_pad_init(float *est, S *dst, const S *src, int fftH, int fftW, int dataH, int dataW, int by, int bx)
{
    GRID_STRIDE(i, (size_t)fftH * fftW)
    {
        const int y = (int)(i / fftW), x = (int)(i % fftW);
        dst[i] = src[(size_t)clamp_src(y, dataH, by) * dataW + clamp_src(x, dataW, bx)];
        est[i] += 10;
    }
}

__global__ void k_unpad32(float *dst, const float *src, int fftW, int dataH, int dataW)
{
    GRID_STRIDE(i, (size_t)dataH * dataW)
    {
        const int y = (int)(i / dataW), x = (int)(i % dataW);
        dst[i] = src[(size_t)y * fftW + x];
    }
}

template <typename S>
__global__ void k_unpad(S *dst, const float *src, int fftW, int dataH, int dataW, float mx)
{
    GRID_STRIDE(i, (size_t)dataH * dataW)
    {
        const int y = (int)(i / dataW), x = (int)(i % dataW);
        float v = src[(size_t)y * fftW + x];
        if (v > mx)
            v = mx;
        dst[i] = (S)__float2uint_rz(v);
    }
}

__global__ void k_modulate(float2 *dst, const float2 *src, size_t n, float c)
{
    GRID_STRIDE(i, n)
    {
        const float2 a = src[i], b = dst[i];
        dst[i] = make_float2(c * (a.x * b.x - a.y * b.y), c * (a.y * b.x + a.x * b.y));
    }
}

__global__ void k_multiply(const float *a, const float *b, const float *w, float *dest, size_t n)
{
    GRID_STRIDE(i, n)
    {
        const float t = a[i] * b[i];
        dest[i] += w[i] * (t - dest[i]);
    }
}

template <typename S>
__global__ void k_divide(const S *a, const float *b, float *dest, size_t n)
{
    GRID_STRIDE(i, n)
    {
        const float q = b[i];
        if (q > 1)
            dest[i] = a[i] / q;
    }
}

} // namespace

extern "C" {

void padKernel(float *d_Dst, float *d_Src, int fftH, int fftW, int kernelH, int kernelW, cudaStream_t s)
{
    k_pad_kernel<<<grid_for((size_t)kernelH * kernelW), 256, 0, s>>>(d_Dst, d_Src, fftH, fftW, kernelH, kernelW);
    FMVD_CHECK(cudaGetLastError());
}

void padWeights(float *d_PaddedWeights, float *d_PaddedWeightSums, float *d_Weights, int fftH, int fftW, int dataH,
                int dataW, int kernelH, int kernelW, cudaStream_t s)
{
    k_pad_weights<<<grid_for((size_t)fftH * fftW), 256, 0, s>>>(d_PaddedWeights, d_PaddedWeightSums, d_Weights, fftH,
                                                               fftW, dataH, dataW, kernelH / 2, kernelW / 2);
    FMVD_CHECK(cudaGetLastError());
}

void normalizeWeights(float *d_PaddedWeights, float *d_PaddedWeightSums, int fftH, int fftW, cudaStream_t s)
{
    k_normalize_weights<<<grid_for((size_t)fftH * fftW), 256, 0, s>>>(d_PaddedWeights, d_PaddedWeightSums,
                                                                     (size_t)fftH * fftW);
    FMVD_CHECK(cudaGetLastError());
}

void padDataClampToBorder32(float *d_PaddedData, float *d_Data, int fftH, int fftW, int dataH, int dataW, int kernelH,
                            int kernelW, cudaStream_t s)
{
    k_pad_clamp<float><<<grid_for((size_t)fftH * fftW), 256, 0, s>>>(d_PaddedData, d_Data, fftH, fftW, dataH, dataW,
                                                                     kernelH / 2, kernelW / 2);
    FMVD_CHECK(cudaGetLastError());
}

void unpadData32(float *d_Dst, float *d_Src, int fftH, int fftW, int dataH, int dataW, cudaStream_t s)
{
    (void)fftH;
    k_unpad32<<<grid_for((size_t)dataH * dataW), 256, 0, s>>>(d_Dst, d_Src, fftW, dataH, dataW);
    FMVD_CHECK(cudaGetLastError());
}

void modulateAndNormalize(fComplex *d_Dst, fComplex *d_Src, int fftH, int fftW, int padding, cudaStream_t s)
{
    const size_t n = (size_t)fftH * (fftW / 2 + padding);
    k_modulate<<<grid_for(n), 256, 0, s>>>((float2 *)d_Dst, (const float2 *)d_Src, n, 1.0f / (float)(fftW * fftH));
    FMVD_CHECK(cudaGetLastError());
}

void multiply32(float *d_a, float *d_b, float *d_weights, float *d_dest, int fftH, int fftW, cudaStream_t s)
{
    const size_t n = (size_t)fftH * fftW;
    k_multiply<<<grid_for(n), 256, 0, s>>>(d_a, d_b, d_weights, d_dest, n);
    FMVD_CHECK(cudaGetLastError());
}

#define FMVD_SAMPLE_LAUNCHERS(S, N, MAXV)                                                                              \
    void padDataClampToBorderAndInitialize_##N(float *d_estimate, S *d_Dst, S *d_Src, float *d_Weights, int fftH,      \
                                               int fftW, int dataH, int dataW, int p9, int p10, cudaStream_t s)        \
    {                                                                                                                  \
        (void)d_Weights;                                                                                               \
        k_pad_init<S><<<grid_for((size_t)fftH * fftW), 256, 0, s>>>(d_estimate, d_Dst, d_Src, fftH, fftW, dataH,       \
                                                                    dataW, p10 / 2, p9 / 2);                          \
        FMVD_CHECK(cudaGetLastError());                                                                                \
    }                                                                                                                  \
    void unpadData_##N(S *d_Data, float *d_PaddedData, int fftH, int fftW, int dataH, int dataW, cudaStream_t s)      \
    {                                                                                                                  \
        (void)fftH;                                                                                                    \
        k_unpad<S><<<grid_for((size_t)dataH * dataW), 256, 0, s>>>(d_Data, d_PaddedData, fftW, dataH, dataW, MAXV);    \
        FMVD_CHECK(cudaGetLastError());                                                                                \
    }                                                                                                                  \
    void divide_##N(S *d_a, float *d_b, float *d_dest, int fftH, int fftW, cudaStream_t s)                           \
    {                                                                                                                  \
        const size_t n = (size_t)fftH * fftW;                                                                          \
        k_divide<S><<<grid_for(n), 256, 0, s>>>(d_a, d_b, d_dest, n);                                                  \
        FMVD_CHECK(cudaGetLastError());                                                                                \
    }

FMVD_SAMPLE_LAUNCHERS(unsigned short, 16, 65535.f)
FMVD_SAMPLE_LAUNCHERS(unsigned char, 8, 255.f)

} // extern "C"
