// Fused per-plane Richardson-Lucy passes on sm_100a.
//
// One RL view update of the reference (fmvd_deconvolve.impl.cpp:264-272:
// R2C, modulate, C2R, divide, R2C, modulate, C2R, multiply32 = 4 FFTs and 4
// element-wise sweeps, 8 launches per plane) becomes four launches over a
// whole batch of plane pairs:
//
//   row pass  "divide": inverse row FFT of the blurred estimate, the data/blur
//             ratio (the reference's q > 1 rule), forward row FFT of the ratio
//   col pass : forward column FFT, times the view's kernel-2 spectrum,
//             inverse column FFT
//   row pass  "update": inverse row FFT (correction r), the weighted
//             multiplicative update e += w (e r - e), forward row FFT of the
//             new estimate (or, after the last update, the cropped, clipped,
//             truncated sample output)
//   col pass : forward column FFT, times the next view's kernel-1 spectrum,
//             inverse column FFT
//
// Two real planes share one complex transform (real part = plane 2p,
// imaginary part = plane 2p+1): convolution with a real kernel acts on both
// parts independently, so every FFT does the work of two real transforms.
// Each pass keeps its lines in shared memory and registers; between passes
// the batch's complex planes are the only traffic, sized by the host to stay
// resident in L2.
#include "fft_engine.cuh"
#include "rl_kernels.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <vector>

namespace fmvd {

// Kernel launches issued by this library (host-side count, for reporting).
static unsigned long long g_launches = 0;
unsigned long long rl_launch_count() { return g_launches; }
void rl_count_launch(unsigned long long n) { g_launches += n; }

// Work-plane tiling: 2 rows x 8 columns of complex (128 bytes) per tile.
constexpr int kTR = 2;
constexpr int kTC = 8;

__host__ __device__ __forceinline__ size_t tile_index(int y, int x, int W)
{
    return (size_t)(y >> 1) * (2 * W) + (size_t)(x >> 3) * 16 + (y & 1) * 8 + (x & 7);
}

__device__ __forceinline__ int clamp_src(int i, int n, int border)
{
    return i < n ? i : (i < n + border ? n - 1 : 0);
}

// Rows per row-pass block and columns per column-pass block.
__host__ __device__ constexpr int row_f(int W) { return W <= 1024 ? 2048 / W : 2; }
__host__ __device__ constexpr int col_f(int H) { return H <= 256 ? 2048 / H : (H <= 1024 ? 8 : 4); }
constexpr int kE = 16;  // complex values per thread

template <int N, int F>
struct Cfg {
    static constexpr int NT = F * N / kE;
    static constexpr size_t smem = 2 * sizeof(float) * SmemLayout<N>::floats(F);
};

// ----------------------------------------------------------- row passes
enum RowMode { ROW_INIT = 0, ROW_DIVIDE = 1, ROW_UPDATE = 2 };

struct RowArgs {
    RlDims d;
    RlBatch b;
    const float2 *tw;
    int view;
    int last;
};

template <int W, int F>
__device__ __forceinline__ void load_rows(const float2 *__restrict__ src, float *sre, float *sim)
{
    using L = SmemLayout<W>;
    constexpr int NT = Cfg<W, F>::NT;
    constexpr int units = F * W / 2;  // float4 = two complex
    const float4 *s4 = reinterpret_cast<const float4 *>(src);
#pragma unroll 4
    for (int u = threadIdx.x; u < units; u += NT) {
        const int l = 2 * u;
        const int yl2 = l / (2 * W), rem = l % (2 * W);
        const int yl = 2 * yl2 + ((rem & 15) >> 3);
        const int x = (rem >> 4) * 8 + (rem & 7);
        const float4 q = s4[u];
        const int a = L::at(yl, x);
        sre[a] = q.x;
        sim[a] = q.y;
        const int a1 = L::at(yl, x + 1);
        sre[a1] = q.z;
        sim[a1] = q.w;
    }
}

template <int W, int F>
__device__ __forceinline__ void store_rows(float2 *__restrict__ dst, const float *sre, const float *sim)
{
    using L = SmemLayout<W>;
    constexpr int NT = Cfg<W, F>::NT;
    constexpr int units = F * W / 2;
    float4 *d4 = reinterpret_cast<float4 *>(dst);
#pragma unroll 4
    for (int u = threadIdx.x; u < units; u += NT) {
        const int l = 2 * u;
        const int yl2 = l / (2 * W), rem = l % (2 * W);
        const int yl = 2 * yl2 + ((rem & 15) >> 3);
        const int x = (rem >> 4) * 8 + (rem & 7);
        const int a = L::at(yl, x), a1 = L::at(yl, x + 1);
        d4[u] = make_float4(sre[a], sim[a], sre[a1], sim[a1]);
    }
}

__device__ __forceinline__ float load_sample(const void *base, size_t idx, int bits)
{
    return bits == 16 ? (float)__ldg(reinterpret_cast<const unsigned short *>(base) + idx)
                      : (float)__ldg(reinterpret_cast<const unsigned char *>(base) + idx);
}

// Float to sample as the reference's unpad kernel: clip at the maximum,
// then convert with truncation (saturating at 0 for negatives).
__device__ __forceinline__ void store_sample(void *base, size_t idx, float v, int bits)
{
    if (bits == 16) {
        if (v > 65535.f) v = 65535.f;
        reinterpret_cast<unsigned short *>(base)[idx] = (unsigned short)__float2uint_rz(v);
    } else {
        if (v > 255.f) v = 255.f;
        reinterpret_cast<unsigned char *>(base)[idx] = (unsigned char)__float2uint_rz(v);
    }
}

template <int W, int F, int MODE>
__global__ void __launch_bounds__(Cfg<W, F>::NT) row_pass(const RowArgs a)
{
    extern __shared__ float smem[];
    float *sre = smem;
    float *sim = smem + SmemLayout<W>::floats(F);
    constexpr int NT = Cfg<W, F>::NT;
    using EG = Edge<W, F, NT>;
    const RlDims &d = a.d;
    const int p = blockIdx.y;
    const int y0 = blockIdx.x * F;
    const int H = d.H;
    float2 *C = a.b.C + (size_t)p * H * W + (size_t)y0 * W;
    float2 v[EG::E];

    if (MODE != ROW_INIT) {
        load_rows<W, F>(C, sre, sim);
        __syncthreads();
        fft<W, F, NT, +1, false>(sre, sim, v, a.tw);
    }

    const int z0 = 2 * p, z1 = 2 * p + 1;
    const bool has1 = z1 < a.b.nplanes;
    float2 *est = a.b.est + (size_t)p * H * W;

    if (MODE == ROW_INIT) {
        const float e0 = a.b.init_value, e1 = has1 ? a.b.init_value : 0.f;
#pragma unroll
        for (int e = 0; e < EG::E; e++) {
            int f, x;
            EG::pos(e, f, x);
            v[e] = make_float2(e0, e1);
            est[(size_t)(y0 + f) * W + x] = v[e];
        }
    } else if (MODE == ROW_DIVIDE) {
        const size_t vb = (size_t)a.view * a.b.view_stride;
        const size_t o0 = vb + (size_t)z0 * a.b.plane_stride;
        const size_t o1 = vb + (size_t)(has1 ? z1 : z0) * a.b.plane_stride;
#pragma unroll
        for (int e = 0; e < EG::E; e++) {
            int f, x;
            EG::pos(e, f, x);
            const int sy = clamp_src(y0 + f, d.dataH, d.byD);
            const int sx = clamp_src(x, d.dataW, d.bxD);
            const size_t si = (size_t)sy * d.dataW + sx;
            float2 q = v[e];
            if (q.x > 1.f)
                q.x = load_sample(a.b.data, o0 + si, d.bits) / q.x;
            if (q.y > 1.f)
                q.y = has1 ? load_sample(a.b.data, o1 + si, d.bits) / q.y : 0.f;
            v[e] = q;
        }
    } else {  // ROW_UPDATE
        const float *wv = a.b.weights + (size_t)a.view * d.dataH * d.dataW;
#pragma unroll
        for (int e = 0; e < EG::E; e++) {
            int f, x;
            EG::pos(e, f, x);
            const int y = y0 + f;
            const float w = __ldg(wv + (size_t)clamp_src(y, d.dataH, d.byW) * d.dataW + clamp_src(x, d.dataW, d.bxW));
            const size_t ei = (size_t)y * W + x;
            float2 c = est[ei];
            const float2 r = v[e];
            c.x += w * (c.x * r.x - c.x);
            c.y += w * (c.y * r.y - c.y);
            est[ei] = c;
            v[e] = c;
            if (a.last && y < d.dataH && x < d.dataW) {
                store_sample(a.b.out, (size_t)z0 * a.b.plane_stride + (size_t)y * d.dataW + x, c.x, d.bits);
                if (has1)
                    store_sample(a.b.out, (size_t)z1 * a.b.plane_stride + (size_t)y * d.dataW + x, c.y, d.bits);
            }
        }
        if (a.last)
            return;
    }

    fft<W, F, NT, -1, true>(sre, sim, v, a.tw);
    regs_to_smem<W, F, NT>(sre, sim, v);
    __syncthreads();
    store_rows<W, F>(C, sre, sim);
}

// --------------------------------------------------------- column pass
struct ColArgs {
    float2 *C;
    const float2 *spec;  // column-pass launch layout
    const float2 *tw;
    int H, W;
};

template <int H, int F>
__global__ void __launch_bounds__(Cfg<H, F>::NT) col_pass(const ColArgs a)
{
    extern __shared__ float smem[];
    float *sre = smem;
    float *sim = smem + SmemLayout<H>::floats(F);
    constexpr int NT = Cfg<H, F>::NT;
    using EG = Edge<H, F, NT>;
    using L = SmemLayout<H>;
    const int W = a.W;
    const int p = blockIdx.y;
    const int x0 = blockIdx.x * F;
    float2 *C = a.C + (size_t)p * H * W;

    // load F columns: units of two complex along x
    constexpr int units = H * F / 2;
#pragma unroll 4
    for (int u = threadIdx.x; u < units; u += NT) {
        const int c2 = u % (F / 2), y = u / (F / 2);
        const int x = x0 + 2 * c2;
        const float4 q = *reinterpret_cast<const float4 *>(C + tile_index(y, x, W));
        const int a0 = L::at(2 * c2, y), a1 = L::at(2 * c2 + 1, y);
        sre[a0] = q.x;
        sim[a0] = q.y;
        sre[a1] = q.z;
        sim[a1] = q.w;
    }
    __syncthreads();

    float2 v[EG::E];
    fft<H, F, NT, -1, false>(sre, sim, v, a.tw);
    const float2 *sp = a.spec + (size_t)blockIdx.x * EG::E * NT + threadIdx.x;
#pragma unroll
    for (int e = 0; e < EG::E; e++)
        v[e] = cmul(v[e], __ldg(sp + (size_t)e * NT));
    fft<H, F, NT, +1, true>(sre, sim, v, a.tw);
    regs_to_smem<H, F, NT>(sre, sim, v);
    __syncthreads();
#pragma unroll 4
    for (int u = threadIdx.x; u < units; u += NT) {
        const int c2 = u % (F / 2), y = u / (F / 2);
        const int x = x0 + 2 * c2;
        const int a0 = L::at(2 * c2, y), a1 = L::at(2 * c2 + 1, y);
        *reinterpret_cast<float4 *>(C + tile_index(y, x, W)) = make_float4(sre[a0], sim[a0], sre[a1], sim[a1]);
    }
}

__global__ void write_estimate_kernel(const RlDims d, const RlBatch b)
{
    const size_t plane = (size_t)d.dataH * d.dataW;
    const size_t total = plane * b.nplanes;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(i / plane);
        const int y = (int)((i % plane) / d.dataW), x = (int)(i % d.dataW);
        const float2 e = b.est[(size_t)(z >> 1) * d.H * d.W + (size_t)y * d.W + x];
        store_sample(b.out, i, (z & 1) ? e.y : e.x, d.bits);
    }
}

__global__ void split_estimate_kernel(const float2 *__restrict__ est, int nplanes, size_t plane, float *__restrict__ out)
{
    const size_t total = plane * nplanes;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t z = i / plane, r = i % plane;
        const float2 e = est[(z >> 1) * plane + r];
        out[i] = (z & 1) ? e.y : e.x;
    }
}

// Column-pass launch layout of a natural-order H x W spectrum: block bx,
// register slot e, thread t -> (row, column) of the edge pattern.
__global__ void permute_spectrum(const double2 *__restrict__ nat, float2 *__restrict__ out, int H, int W, int F,
                                 int NT, int R, double scale)
{
    const int E = kE;
    const size_t total = (size_t)(W / F) * E * NT;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int t = (int)(i % NT);
        const int e = (int)((i / NT) % E);
        const int bx = (int)(i / ((size_t)NT * E));
        const int b = e / R, m = e % R;
        const int q = t + b * NT;
        const int f = q / (H / R);
        const int n = q % (H / R) + m * (H / R);
        const double2 k = nat[(size_t)n * W + (size_t)bx * F + f];
        out[i] = make_float2((float)(k.x * scale), (float)(k.y * scale));
    }
}

// Separable direct DFT of a small kernel placed at (y - kH/2, x - kW/2) mod (H, W).
// Step 1: A[y][v] = sum_x k[y][x] exp(-2 pi i v (x - cx) / W)
__global__ void kspec_rows(const float *__restrict__ k, int kH, int kW, int W, const double2 *__restrict__ twW,
                           double2 *__restrict__ A)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (v >= W)
        return;
    double re = 0, im = 0;
    const int cx = kW / 2;
    for (int x = 0; x < kW; x++) {
        const long long ph = ((long long)v * (x - cx)) % W;
        const double2 t = twW[ph < 0 ? ph + W : ph];
        const double kv = k[y * kW + x];
        re += kv * t.x;
        im += kv * t.y;
    }
    A[(size_t)y * W + v] = make_double2(re, im);
}

// Step 2: K[u][v] = sum_y A[y][v] exp(-2 pi i u (y - cy) / H)
__global__ void kspec_cols(const double2 *__restrict__ A, int kH, int H, int W, const double2 *__restrict__ twH,
                           double2 *__restrict__ K)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int u = blockIdx.y;
    if (v >= W)
        return;
    double re = 0, im = 0;
    const int cy = kH / 2;
    for (int y = 0; y < kH; y++) {
        const long long ph = ((long long)u * (y - cy)) % H;
        const double2 t = twH[ph < 0 ? ph + H : ph];
        const double2 a = A[(size_t)y * W + v];
        re += a.x * t.x - a.y * t.y;
        im += a.x * t.y + a.y * t.x;
    }
    K[(size_t)u * W + v] = make_double2(re, im);
}

__global__ void normalize_weights_kernel(const float *__restrict__ in, float *__restrict__ out, int V, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int v = 0; v < V; v++)
            s += in[(size_t)v * n + i];
        for (int v = 0; v < V; v++) {
            const float w = in[(size_t)v * n + i];
            out[(size_t)v * n + i] = s > 0.f ? w / s : w;
        }
    }
}

__device__ __forceinline__ int clamp_src_d(int i, int n, int border)
{
    return i < n ? i : (i < n + border ? n - 1 : 0);
}

__global__ void conv_same_kernel(const double *__restrict__ img, int dH, int dW, const double *__restrict__ k, int kH,
                                 int kW, int fH, int fW, double *__restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= dW || y >= dH)
        return;
    double acc = 0;
    for (int ky = 0; ky < kH; ky++) {
        int py = (y - (ky - kH / 2)) % fH;
        if (py < 0)
            py += fH;
        const int sy = clamp_src_d(py, dH, kH / 2);
        for (int kx = 0; kx < kW; kx++) {
            int px = (x - (kx - kW / 2)) % fW;
            if (px < 0)
                px += fW;
            const int sx = clamp_src_d(px, dW, kW / 2);
            acc += img[(size_t)sy * dW + sx] * k[ky * kW + kx];
        }
    }
    out[(size_t)y * dW + x] = acc;
}

// ------------------------------------------------------------ dispatch
#define FMVD_FOR_EACH_LENGTH(X) \
    X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(1536) X(2048) X(2560) X(3072) X(3584) X(4096)

bool rl_length_supported(int n)
{
    switch (n) {
#define X(N) case N:
        FMVD_FOR_EACH_LENGTH(X)
#undef X
        return true;
    default:
        return false;
    }
}

int snap_transform_size(int n)
{
    // fmvd_deconvolve.cpp:22-51
    auto align = [](int a, int b) { return (a % b != 0) ? (a - a % b + b) : a; };
    n = align(n, 16);
    int hibit = 31;
    while (hibit >= 0 && !(n & (1u << hibit)))
        hibit--;
    unsigned lo = 1u << hibit;
    if (lo == (unsigned)n)
        return n;
    unsigned hi = 1u << (hibit + 1);
    if (hi <= 1024)
        return (int)hi;
    return align(n, 512);
}

static int sched_edge(int n) { return make_schedule(n).r[0]; }
static int col_f_for(int H, int W);

size_t rl_spectrum_elems(int H, int W)
{
    const int F = col_f_for(H, W);
    const int NT = F * H / kE;
    return (size_t)(W / F) * kE * NT;
}

void rl_upload_constants()
{
    static OddRadixTable t;
    for (int R = 3; R < 32; R += 2)
        for (int k = 0; k < R; k++) {
            t.c[R][k] = (float)cos(2.0 * M_PI * k / R);
            t.s[R][k] = (float)sin(2.0 * M_PI * k / R);
        }
    cudaMemcpyToSymbol(g_odd, &t, sizeof(t));
}

// Dynamic shared memory above 48 KB needs an opt-in per function and device.
template <typename K>
static void configure_smem(K kern, size_t bytes, unsigned &mask)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned bit = 1u << (dev & 31);
    if (!(mask & bit)) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        mask |= bit;
    }
}

// Rows per block: row_f(W) when it divides H, else 2 (tiny planes only).
template <int W, int F, int MODE>
static void launch_row_f(const RowArgs &a, cudaStream_t s)
{
    using C = Cfg<W, F>;
    auto kern = row_pass<W, F, MODE>;
    static unsigned mask = 0;
    configure_smem(kern, C::smem, mask);
    dim3 grid(a.d.H / F, a.b.npairs);
    kern<<<grid, C::NT, C::smem, s>>>(a);
    g_launches++;
}

template <int W, int MODE>
static void launch_row(const RowArgs &a, cudaStream_t s)
{
    constexpr int F = row_f(W);
    if constexpr (F > 2) {
        if (a.d.H % F != 0) {
            launch_row_f<W, 2, MODE>(a, s);
            return;
        }
    }
    launch_row_f<W, F, MODE>(a, s);
}

template <int H, int F>
static void launch_col_f(const ColArgs &a, int npairs, cudaStream_t s)
{
    using C = Cfg<H, F>;
    auto kern = col_pass<H, F>;
    static unsigned mask = 0;
    configure_smem(kern, C::smem, mask);
    dim3 grid(a.W / F, npairs);
    kern<<<grid, C::NT, C::smem, s>>>(a);
    g_launches++;
}

// Columns per block: col_f(H) when it divides W, else 8 (tiny planes only).
static int col_f_for(int H, int W) { return (W % col_f(H) == 0) ? col_f(H) : 8; }

template <int H>
static void launch_col(const ColArgs &a, int npairs, cudaStream_t s)
{
    constexpr int F = col_f(H);
    if constexpr (F > 8) {
        if (a.W % F != 0) {
            launch_col_f<H, 8>(a, npairs, s);
            return;
        }
    }
    launch_col_f<H, F>(a, npairs, s);
}

template <int MODE>
static void dispatch_row(const RowArgs &a, cudaStream_t s)
{
    switch (a.d.W) {
#define X(N) \
    case N: launch_row<N, MODE>(a, s); break;
        FMVD_FOR_EACH_LENGTH(X)
#undef X
    default: break;
    }
}

void rl_init(const RlDims &d, const RlBatch &b, const RlTables &t, cudaStream_t s)
{
    RowArgs a{d, b, t.twW, 0, 0};
    dispatch_row<ROW_INIT>(a, s);
}

void rl_divide(const RlDims &d, const RlBatch &b, const RlTables &t, int view, cudaStream_t s)
{
    RowArgs a{d, b, t.twW, view, 0};
    dispatch_row<ROW_DIVIDE>(a, s);
}

void rl_update(const RlDims &d, const RlBatch &b, const RlTables &t, int view, bool last, cudaStream_t s)
{
    RowArgs a{d, b, t.twW, view, last ? 1 : 0};
    dispatch_row<ROW_UPDATE>(a, s);
}

void rl_col(const RlDims &d, const RlBatch &b, const RlTables &t, const float2 *spectrum, cudaStream_t s)
{
    ColArgs a{b.C, spectrum, t.twH, d.H, d.W};
    switch (d.H) {
#define X(N) \
    case N: launch_col<N>(a, b.npairs, s); break;
        FMVD_FOR_EACH_LENGTH(X)
#undef X
    default: break;
    }
}

void rl_kernel_spectrum(const float *d_kernel, int kH, int kW, int H, int W, const double2 *twH, const double2 *twW,
                        double2 *work, float2 *d_out, cudaStream_t s)
{
    double2 *A = work;
    double2 *K = work + (size_t)kH * W;
    kspec_rows<<<dim3((W + 127) / 128, kH), 128, 0, s>>>(d_kernel, kH, kW, W, twW, A);
    kspec_cols<<<dim3((W + 127) / 128, H), 128, 0, s>>>(A, kH, H, W, twH, K);
    const int F = col_f_for(H, W);
    const int NT = F * H / kE;
    const int R = sched_edge(H);
    const size_t total = rl_spectrum_elems(H, W);
    permute_spectrum<<<(int)((total + 255) / 256 > 4096 ? 4096 : (total + 255) / 256), 256, 0, s>>>(
        K, d_out, H, W, F, NT, R, 1.0 / ((double)H * (double)W));
}

void rl_write_estimate(const RlDims &d, const RlBatch &b, cudaStream_t s)
{
    write_estimate_kernel<<<1024, 256, 0, s>>>(d, b);
    g_launches++;
}

void rl_split_estimate(const RlDims &d, const float2 *est, int nplanes, float *out, cudaStream_t s)
{
    split_estimate_kernel<<<1024, 256, 0, s>>>(est, nplanes, (size_t)d.H * d.W, out);
    g_launches++;
}

void rl_normalize_weights(const float *d_in, float *d_out, int V, size_t n, cudaStream_t s)
{
    int blocks = (int)((n + 255) / 256);
    if (blocks > 4096)
        blocks = 4096;
    normalize_weights_kernel<<<blocks, 256, 0, s>>>(d_in, d_out, V, n);
}

void rl_conv_same(const double *d_img, int dH, int dW, const double *d_k, int kH, int kW, double *d_out,
                  cudaStream_t s)
{
    const int fH = snap_transform_size(dH + kH - 1);
    const int fW = snap_transform_size(dW + kW - 1);
    conv_same_kernel<<<dim3((dW + 127) / 128, dH), 128, 0, s>>>(d_img, dH, dW, d_k, kH, kW, fH, fW, d_out);
}

} // namespace fmvd
