// Per-plane FP64 statistics of estimates (the convergence check) and the
// padding of a data-plane estimate onto the FFT plane (warm starts).
//
// The RL update itself stays in FP32; FP64 is used only here, in the
// intensity-sum reductions that decide whether an iteration count has
// converged: summed in float, a 1024 x 1024 plane of values near 1e3 would
// lose the relative changes of 1e-6 that the check compares.
#include "fmvd_internal.h"
#include "rl_kernels.h"

namespace fmvd {

namespace {

constexpr int kStatThreads = 512;

// One block per plane, fixed reduction order (deterministic).  Per plane p:
// out[4p + 0] = sum a, [1] = sum a^2, [2] = sum (a - b)^2, [3] = sum |a - b|
// over rows < rows and columns < cols of the H x W plane (b null: 0).
__global__ void __launch_bounds__(kStatThreads) plane_stats_kernel(const float *__restrict__ a,
                                                                   const float *__restrict__ b, int H, int W,
                                                                   int rows, int cols, double *__restrict__ out)
{
    const int p = blockIdx.x;
    const size_t base = (size_t)p * H * W;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int nwarps = kStatThreads / 32;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int y = warp; y < rows; y += nwarps) {
        const float *ar = a + base + (size_t)y * W;
        const float *br = b ? b + base + (size_t)y * W : nullptr;
        for (int x = lane; x < cols; x += 32) {
            const double va = (double)__ldg(ar + x);
            s0 += va;
            s1 += va * va;
            if (br) {
                const double dv = va - (double)__ldg(br + x);
                s2 += dv * dv;
                s3 += fabs(dv);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
        s3 += __shfl_down_sync(0xffffffffu, s3, o);
    }
    __shared__ double part[nwarps][4];
    if (lane == 0) {
        part[warp][0] = s0;
        part[warp][1] = s1;
        part[warp][2] = s2;
        part[warp][3] = s3;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0;
        for (int w = 0; w < nwarps; w++)
            t += part[w][threadIdx.x];
        out[4 * (size_t)p + threadIdx.x] = t;
    }
}

__device__ __forceinline__ int clamp_index(int i, int n, int border)
{
    return i < n ? i : (i < n + border ? n - 1 : 0);
}

// Data-plane float estimates (dataH x dataW) onto the H x W FFT plane with
// the clamp-to-border padding the data receives (rows beyond dataH + byD and
// columns beyond dataW + bxD wrap to row / column 0), raised to floor_value
// (the multiplicative RL update needs a positive estimate).
__global__ void pad_estimate_kernel(const float *__restrict__ in, float *__restrict__ out, int H, int W, int dataH,
                                    int dataW, int byD, int bxD, float floor_value)
{
    const int p = blockIdx.z;
    const int y = blockIdx.y;
    const int sy = clamp_index(y, dataH, byD);
    const float *src = in + ((size_t)p * dataH + sy) * dataW;
    float *dst = out + ((size_t)p * H + y) * W;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x)
        dst[x] = fmaxf(__ldg(src + clamp_index(x, dataW, bxD)), floor_value);
}

} // namespace

bool plane_stats(const float *a, const float *b, int nplanes, int H, int W, int rows, int cols, double *out,
                 cudaStream_t s)
{
    if (nplanes <= 0)
        return true;
    plane_stats_kernel<<<nplanes, kStatThreads, 0, s>>>(a, b, H, W, rows, cols, out);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

bool pad_estimate(const float *in, float *out, int nplanes, const RlDims &d, float floor_value, cudaStream_t s)
{
    if (nplanes <= 0)
        return true;
    const int threads = 256;
    const int chunk = 65535;  // grid z limit
    for (int p0 = 0; p0 < nplanes; p0 += chunk) {
        const int n = nplanes - p0 < chunk ? nplanes - p0 : chunk;
        const dim3 grid((d.W + threads - 1) / threads, d.H, n);
        pad_estimate_kernel<<<grid, threads, 0, s>>>(in + (size_t)p0 * d.dataH * d.dataW,
                                                     out + (size_t)p0 * d.H * d.W, d.H, d.W, d.dataH, d.dataW,
                                                     d.byD, d.bxD, floor_value);
        rl_count_launch(1);
    }
    return FMVD_CHECK(cudaGetLastError());
}

} // namespace fmvd
