// Host-side interface of the fused Richardson-Lucy pass kernels.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace fmvd {

// Geometry of one plan.  The padded (FFT) plane is H x W; the data plane is
// dataH x dataW.  Padded data uses borders (byD rows, bxD columns) and padded
// weights (byW, bxW): the reference pads data with (kW/2, kH/2) and weights
// with (kH/2, kW/2).
struct RlDims {
    int H, W;
    int dataH, dataW;
    int V;
    int bits;            // 8 or 16 (sample type of data and output)
    int byD, bxD;
    int byW, bxW;
    int col_warps;       // column-pass warps per block (warp engine, H <= 1024)
    int radix_step;      // lines above 1024: kRadixDft or kRadixSums
};

// Schedules of the radix-R step of lines above 1024 (same transform): R-point
// DFTs per position in shared memory, or each group's weighted sum over the
// R sub-lines.
constexpr int kRadixDft = 1;
constexpr int kRadixSums = 2;

// One batch of plane pairs resident on the device.  Pair p packs planes
// 2p (real part) and 2p+1 (imaginary part).
struct RlBatch {
    float2 *C;            // npairs x H x W complex work planes, tiled 2 x 8
    float2 *est;          // npairs x H x W (estimate of plane 2p, of plane 2p+1)
    const void *data;     // view v, plane z at data + (v * view_stride + z * plane_stride) samples
    size_t view_stride;
    size_t plane_stride;  // dataH * dataW
    const float *weights; // V x dataH x dataW, normalised over views
    void *out;            // nplanes x dataH x dataW samples
    int npairs;
    int nplanes;
    float init_value;     // 10 * V
    const float *init;    // optional initial estimate: nplanes x H x W floats (null: init_value everywhere)
    int *status;          // set to 1 by a kernel whose bulk copy wait timed out
};

// Per-plan constants that the kernels read.
struct RlTables {
    const float2 *twH;   // exp(-2 pi i n / H)            (lengths above 1024)
    const float2 *twW;   // exp(-2 pi i n / W)
    const float2 *wtwH;  // warp-FFT twiddles of H (of kLineM above 1024; layout in warp_twiddles)
    const float2 *wtwW;  // warp-FFT twiddles of W
};

// Lanes per line of the warp FFT for length n (0 when n > 1024).
int rl_warp_lanes(int n);
// Lines longer than 1024 (R x kLineM, R = 3..8) are split into R sub-lines
// of this length.
constexpr int kLineM = 512;
// Twiddle run of the warp FFT: lane t forms w_N^(t k1), k1 = R j + b, as the
// table entry w_N^(R j t) times (w_N^t)^b, b < R (R = min(E, this)).
constexpr int kWarpTwiddleRun = 2;
// float2 entries of the warp-FFT twiddle table of length n (at least n).
int rl_warp_twiddle_entries(int n);
// Column-pass warps per block for an H x W plane: 'requested' (2, 4 or 8)
// when the plane allows it, the widest allowed when 0, -1 when not allowed.
int rl_col_warps(int H, int W, int requested);

bool rl_length_supported(int n);
// Number of kernel launches this library has issued (all kernels).
unsigned long long rl_launch_count();
void rl_count_launch(unsigned long long n);
// Number of complex values of a column-pass kernel spectrum in its launch layout.
size_t rl_spectrum_elems(int H, int W);

void rl_init(const RlDims &d, const RlBatch &b, const RlTables &t, cudaStream_t s);
void rl_col(const RlDims &d, const RlBatch &b, const RlTables &t, const float2 *spectrum, cudaStream_t s);
void rl_divide(const RlDims &d, const RlBatch &b, const RlTables &t, int view, cudaStream_t s);
void rl_update(const RlDims &d, const RlBatch &b, const RlTables &t, int view, bool last, cudaStream_t s);

// Cropped, clipped, truncated samples of the current estimate (used when no
// iteration runs: the output is then the initial estimate).
void rl_write_estimate(const RlDims &d, const RlBatch &b, cudaStream_t s);
// Float estimates of nplanes planes (H x W each) from the pair layout.
void rl_split_estimate(const RlDims &d, const float2 *est, int nplanes, float *out, cudaStream_t s);

// Plan-time helpers (device work in FP32, launched on stream s).
// Kernel spectrum of a kH x kW kernel centred at (kH/2, kW/2) -> (0, 0) on the
// H x W plane, scaled by 1 / (H W), in the column-pass launch layout.
// twH / twW: exp(-2 pi i n / N) tables; work must hold H * W + kH * W complex
// floats.  col_warps: the plan's column-pass warps (the launch layout depends
// on it).
void rl_kernel_spectrum(const float *d_kernel, int kH, int kW, int H, int W, const float2 *twH, const float2 *twW,
                        float2 *work, float2 *d_out, int col_warps, cudaStream_t s);
// Weights normalised over views where the sum is positive.
void rl_normalize_weights(const float *d_in, float *d_out, int V, size_t n, cudaStream_t s);
// Clamp-to-border padded circular convolution of a dH x dW image with a
// kH x kW kernel on the snapTransformSize domain, cropped to dH x dW.
void rl_conv_same(const float *d_img, int dH, int dW, const float *d_k, int kH, int kW, float *d_out, cudaStream_t s);

int snap_transform_size(int n);

} // namespace fmvd
