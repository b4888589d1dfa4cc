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
#include "warp_fft.cuh"
#include "tma_util.cuh"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <type_traits>
#include <vector>

namespace fmvd {

// Kernel launches issued by this library (host-side count, for reporting).
static unsigned long long g_launches = 0;
unsigned long long rl_launch_count() { return g_launches; }
void rl_count_launch(unsigned long long n) { g_launches += n; }

// Work planes are row-major (natural order): element (y, x) of pair p at
// C[(p * H + y) * W + x].  Column blocks read runs of 4 to 8 complex values
// (32 to 64 bytes, whole L2 sectors) per row.
__host__ __device__ __forceinline__ size_t tile_index(int y, int x, int W) { return (size_t)y * W + x; }

__device__ __forceinline__ int clamp_src(int i, int n, int border)
{
    // i < n: i; n <= i < n + border: n - 1; beyond: 0 (i >= 0)
    const int c = min(i, n - 1);
    return i < n + border ? c : 0;
}

// Programmatic dependent launch.  Every pass lets the next kernel of its
// stream launch as soon as all of its own blocks have started
// (launch_dependents), and waits for the previous kernel to complete, with
// its writes visible, before it reads anything an earlier kernel produced
// (dependency_wait).  Work on constant operands (weights, spectra) may run
// before the wait, so the next pass's blocks set up while the tail of the
// previous one finishes.  Launched without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Requests the 128-byte line holding p into L1 (no result, no wait).
__device__ __forceinline__ void prefetch_l1(const void *p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Shared-memory loads by 32-bit shared-window address.
__device__ __forceinline__ float lds_f32(uint32_t addr)
{
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ float2 lds_f32x2(uint32_t addr)
{
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
    return v;
}
template <int BITS>
__device__ __forceinline__ float lds_sample(uint32_t row, int sx)
{
    uint32_t v;
    if constexpr (BITS == 16)
        asm volatile("ld.shared.u16 %0, [%1];" : "=r"(v) : "r"(row + 2u * sx) : "memory");
    else
        asm volatile("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(row + (uint32_t)sx) : "memory");
    return (float)v;
}

// ----------------------------------------------------------- row passes
enum RowMode { ROW_INIT = 0, ROW_DIVIDE = 1, ROW_UPDATE = 2 };

struct RowArgs {
    RlDims d;
    RlBatch b;
    const float2 *tw;
    int view;
    int last;
    int bulk_data;      // data rows may be fetched with 16-byte bulk copies
    int bulk_weights;   // weight rows may be fetched with 16-byte bulk copies
    int group_floats;   // warp engine: shared floats per group (transpose + prefetch)
    const float2 *twN;  // lines above 1024: exp(-2 pi i n / W), n < W
};

// Sample loads and estimate traffic are streamed (evict-first in L2) so that
// the batch's complex work planes stay resident in L2 between passes.
__device__ __forceinline__ float load_sample(const void *base, size_t idx, int bits)
{
    return bits == 16 ? (float)__ldcs(reinterpret_cast<const unsigned short *>(base) + idx)
                      : (float)__ldcs(reinterpret_cast<const unsigned char *>(base) + idx);
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

// Element-wise work of the row passes on row y of pair p (row-invariant
// pointers computed once):
//   INIT:   estimate = 10 * nViews (imaginary part 0 for a missing second plane)
//   DIVIDE: blur b -> data / b where b > 1, else b (divide_kernel, the
//           reference's in-place quirk)
//   UPDATE: correction r -> e + w (e r - e) (multiply32_kernel); after the
//           last view of the last iteration also the output samples
// BITS: the sample width when fixed at compile time (8 or 16), else 0.  With
// it fixed, operand rows are read through generic pointers that may point to
// shared or global memory, so the element-wise step has no per-element
// branches.  NOOUT: an update pass known at compile time not to be the last
// one, so the output-sample code is left out.  SMEM (with BITS fixed): the
// operand rows are in shared memory at the s_* addresses (the data rows in
// the divide pass; the weight row in the update pass, and the estimate row
// too when EST_S).
template <int MODE, int BITS = 0, bool NOOUT = false, bool SMEM = false, bool EST_S = SMEM>
struct RowWork {
    const RlDims &d;
    float2 *est;             // row y of the pair's estimate (global)
    const float2 *est_s;     // the same row prefetched into shared memory, or null
    const void *src0, *src1; // data rows (clamped) of planes 2p and 2p+1, view a.view
    bool src_s;              // data rows are in shared memory
    const float *wrow;       // weight row (clamped)
    bool w_s;                // weight row is in shared memory
    void *out0, *out1;       // output rows, or null
    bool has1;
    float init0, init1;
    const float *initr0, *initr1;  // rows of a given initial estimate, or null
    uint32_t s_src0, s_src1, s_w, s_est;  // shared-memory rows (SMEM)

    __device__ __forceinline__ RowWork(const RowArgs &a, int p, int y) : d(a.d)
    {
        const int W = d.W;
        has1 = 2 * p + 1 < a.b.nplanes;
        est = a.b.est + ((size_t)p * d.H + y) * W;
        est_s = nullptr;
        init0 = a.b.init_value;
        init1 = has1 ? a.b.init_value : 0.f;
        initr0 = initr1 = nullptr;
        if (MODE == ROW_INIT && a.b.init) {
            initr0 = a.b.init + ((size_t)(2 * p) * d.H + y) * W;
            initr1 = has1 ? a.b.init + ((size_t)(2 * p + 1) * d.H + y) * W : nullptr;
        }
        const size_t es = d.bits == 16 ? 2 : 1;
        src0 = src1 = nullptr;
        src_s = w_s = false;
        wrow = nullptr;
        out0 = out1 = nullptr;
        if (MODE == ROW_DIVIDE) {
            const size_t base = (size_t)a.view * a.b.view_stride + (size_t)clamp_src(y, d.dataH, d.byD) * d.dataW;
            src0 = (const char *)a.b.data + (base + (size_t)(2 * p) * a.b.plane_stride) * es;
            src1 = has1 ? (const char *)a.b.data + (base + (size_t)(2 * p + 1) * a.b.plane_stride) * es : src0;
        }
        if (MODE == ROW_UPDATE) {
            wrow = a.b.weights + (size_t)a.view * d.dataH * d.dataW + (size_t)clamp_src(y, d.dataH, d.byW) * d.dataW;
            if (a.last && y < d.dataH) {
                out0 = (char *)a.b.out + ((size_t)(2 * p) * a.b.plane_stride + (size_t)y * d.dataW) * es;
                if (has1)
                    out1 = (char *)a.b.out + ((size_t)(2 * p + 1) * a.b.plane_stride + (size_t)y * d.dataW) * es;
            }
        }
    }

    __device__ __forceinline__ float sample(const void *row, int sx) const
    {
        if constexpr (BITS == 16)
            return (float)reinterpret_cast<const unsigned short *>(row)[sx];
        else if constexpr (BITS == 8)
            return (float)reinterpret_cast<const unsigned char *>(row)[sx];
        if (src_s)
            return d.bits == 16 ? (float)reinterpret_cast<const unsigned short *>(row)[sx]
                                : (float)reinterpret_cast<const unsigned char *>(row)[sx];
        return load_sample(row, sx, d.bits);
    }

    __device__ __forceinline__ void apply(int x, float2 &v) const
    {
        if (MODE == ROW_INIT) {
            v = initr0 ? make_float2(__ldcs(initr0 + x), initr1 ? __ldcs(initr1 + x) : 0.f)
                       : make_float2(init0, init1);
            __stcs(est + x, v);
        } else if (MODE == ROW_DIVIDE) {
            // q > 1 keeps the divisor in the range where the fast division is
            // within 2 ulp of the IEEE quotient
            const int sx = clamp_src(x, d.dataW, d.bxD);
            float a0, a1;
            if constexpr (SMEM) {
                a0 = lds_sample<BITS>(s_src0, sx);
                const float s1 = lds_sample<BITS>(s_src1, sx);
                a1 = has1 ? s1 : 0.f;
            } else {
                a0 = sample(src0, sx);
                a1 = has1 ? sample(src1, sx) : 0.f;
            }
            float2 q = v;
            q.x = q.x > 1.f ? __fdividef(a0, q.x) : q.x;
            q.y = q.y > 1.f ? __fdividef(a1, q.y) : q.y;
            v = q;
        } else {
            const int sx = clamp_src(x, d.dataW, d.bxW);
            float w;
            float2 c;
            if constexpr (SMEM) {
                w = lds_f32(s_w + 4u * sx);
                if constexpr (EST_S)
                    c = lds_f32x2(s_est + 8u * x);
                else
                    c = est[x];
            } else if constexpr (BITS != 0) {
                w = wrow[sx];
                c = (est_s ? est_s : est)[x];
            } else {
                w = w_s ? wrow[sx] : __ldg(wrow + sx);
                c = est_s ? est_s[x] : __ldcs(est + x);
            }
            const float2 r = v;
            c.x += w * (c.x * r.x - c.x);
            c.y += w * (c.y * r.y - c.y);
            __stcs(est + x, c);
            v = c;
            if (!NOOUT && out0 && x < d.dataW) {
                store_sample(out0, x, c.x, BITS ? BITS : d.bits);
                if (out1)
                    store_sample(out1, x, c.y, BITS ? BITS : d.bits);
            }
        }
    }
};

// Row pass for W <= 1024: one group of T lanes per row, warp FFT, no block
// synchronisation.  Rows beyond H (only for tiny planes) compute on row H-1
// and store nothing.
// Occupancy knobs of the warp-engine passes (blocks per SM the register
// allocation must allow, and the widest column block).
#ifndef FMVD_ROW_MIN_BLOCKS
#define FMVD_ROW_MIN_BLOCKS 4
#endif
#ifndef FMVD_COL_MIN_BLOCKS
#define FMVD_COL_MIN_BLOCKS 2
#endif
#ifndef FMVD_COL_MAX_WARPS
#define FMVD_COL_MAX_WARPS 8
#endif
constexpr int kRowWarps = 4;

template <int W, int MODE, int BITS, bool NOOUT, bool SMEM>
__global__ void __launch_bounds__(kRowWarps * 32, FMVD_ROW_MIN_BLOCKS) row_pass_w(const RowArgs a)
{
    using WF = WarpFft<W>;
    constexpr int T = WF::T, E = WF::E, G = 32 / T;
    extern __shared__ __align__(16) float smem[];
    __shared__ __align__(8) uint64_t bars[kRowWarps * G];
    __shared__ __align__(8) uint64_t ebars[MODE == ROW_UPDATE ? kRowWarps * G : 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / T, t = lane % T;
    const int gi = warp * G + g;
    float *gbase = smem + (size_t)gi * a.group_floats;
    float2 *tbuf = reinterpret_cast<float2 *>(gbase);                // padded transpose buffer
    char *pf = reinterpret_cast<char *>(gbase + WF::padded_floats);  // prefetch area, 16-byte aligned
    const int H = a.d.H;
    const int yr = blockIdx.x * (kRowWarps * G) + warp * G + g;
    const bool valid = yr < H;
    const int y = valid ? yr : H - 1;
    const int p = blockIdx.y;
    float2 *row = a.b.C + ((size_t)p * H + y) * W;
    RowWork<MODE, BITS, NOOUT, SMEM> work(a, p, y);

    // Rows the element-wise step needs are fetched by the bulk-copy engine
    // while the inverse transform runs: the weight row in the update pass,
    // the two data rows in the divide pass.  The update pass's estimate row
    // lands in the transpose buffer itself, issued once the inverse
    // transform has read its transpose back, so it takes no shared memory
    // of its own.
    // SMEM is set exactly when the launch allows the bulk copies (weights in
    // the update pass, data in the divide pass)
    constexpr bool prefetch = SMEM && MODE != ROW_INIT;
    uint64_t *bar = &bars[gi];
    uint64_t *ebar = &ebars[MODE == ROW_UPDATE ? gi : 0];
    pdl_launch_dependents();
    if (prefetch || MODE == ROW_UPDATE) {
        if (t == 0) {
            mbar_init(bar, 1);
            if (MODE == ROW_UPDATE)
                mbar_init(ebar, 1);
            mbar_fence_init();
        }
        __syncwarp();
    }
    if (prefetch && MODE == ROW_UPDATE && t == 0) {
        // the weight row is a plan constant: requested before the wait
        const uint32_t wb = a.d.dataW * sizeof(float);
        mbar_arrive_expect_tx(bar, wb);
        bulk_load(pf, work.wrow, wb, bar);
    }
    pdl_wait();
    if (prefetch && MODE == ROW_DIVIDE && t == 0) {
        const int es = a.d.bits == 16 ? 2 : 1;
        const uint32_t rb = a.d.dataW * es;
        const uint32_t rs = (rb + 15) & ~15u;
        mbar_arrive_expect_tx(bar, work.has1 ? 2 * rb : rb);
        bulk_load(pf, work.src0, rb, bar);
        if (work.has1)
            bulk_load(pf + rs, work.src1, rb, bar);
    }

    // One copy of the transform code serves both directions: the inverse is
    // conj(DFT(conj(x))), so pass 0 (inverse of the loaded row) and pass 1
    // (forward) run the same loop body; keeping it rolled halves the code the
    // instruction cache must hold.
    float2 v[E];
    if (MODE == ROW_INIT) {
#pragma unroll
        for (int m = 0; m < E; m++)
            v[m] = make_float2(0.f, 0.f);
        if (valid) {
#pragma unroll
            for (int m = 0; m < E; m++)
                work.apply(t + T * m, v[m]);
        }
    }
    int pass = MODE == ROW_INIT ? 1 : 0;
    const auto estimate_to_tbuf = [&]() {
        if (MODE == ROW_UPDATE && pass == 0 && t == 0) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(ebar, W * sizeof(float2));
            bulk_load(tbuf, work.est, W * sizeof(float2), ebar);
        }
    };
#pragma unroll 1
    for (; pass < 2; pass++) {
        if (pass == 0) {
#pragma unroll
            for (int m = 0; m < E; m++) {
                const float2 x = row[t + T * m];
                v[m] = make_float2(x.x, -x.y);
            }
        }
        WF::template run_padded<-1>(v, a.tw, tbuf, t, estimate_to_tbuf);
        if (pass == 1)
            break;
#pragma unroll
        for (int m = 0; m < E; m++)
            v[m].y = -v[m].y;
    if (MODE == ROW_UPDATE) {
        const bool ok_w = !prefetch || mbar_wait(bar, 0);
        const bool ok_e = mbar_wait(ebar, 0);
        if (!ok_w || !ok_e) {
            // a copy did not land in time: flag it (the host reports the
            // batch as failed), wait once more so no copy is left in flight,
            // and continue from global memory where the code allows it
            if (t == 0)
                atomicExch(a.b.status, 1);
            if (!ok_w)
                mbar_wait(bar, 0);
            if (!ok_e)
                mbar_wait(ebar, 0);
        }
        if constexpr (SMEM) {
            work.s_est = smem_u32addr(tbuf);
            work.s_w = smem_u32addr(pf);
        } else if (ok_w && ok_e) {
            work.est_s = tbuf;
            if (prefetch) {
                work.wrow = reinterpret_cast<const float *>(pf);
                work.w_s = true;
            }
        }
    } else if (prefetch) {
        if (!mbar_wait(bar, 0)) {
            // the copy did not land in time: flag it (the host reports the
            // batch as failed) and wait once more so no copy is left in flight
            if (t == 0)
                atomicExch(a.b.status, 1);
            mbar_wait(bar, 0);
        }
        const int es = a.d.bits == 16 ? 2 : 1;
        const uint32_t rs = (a.d.dataW * es + 15) & ~15u;
        work.s_src0 = smem_u32addr(pf);
        work.s_src1 = work.has1 ? smem_u32addr(pf + rs) : work.s_src0;
    }
    if (valid) {
#pragma unroll
        for (int m = 0; m < E; m++)
            work.apply(t + T * m, v[m]);
    }
    if (MODE == ROW_UPDATE && !NOOUT && a.last)
        return;
    if (MODE == ROW_UPDATE)
        __syncwarp();  // the estimate row in tbuf is read before the forward transform writes it
    }
    if (valid) {
#pragma unroll
        for (int m = 0; m < E; m++)
            row[t + T * m] = v[m];
    }
}

// --------------------------------------------------------- column pass
struct ColArgs {
    float2 *C;
    const float2 *spec;  // column-pass launch layout
    const float2 *tw;    // warp-FFT twiddles (of kLineM above 1024)
    int H, W;
    const float2 *twN;   // columns above 1024: exp(-2 pi i n / H), n < H
};

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

// Column tile of the warp engine in shared memory: element (y, c) of the
// block's FC columns.  With 32-lane groups the tile is dense and XOR-swizzled,
// (y, c) at y * FC + (c ^ ((y >> SH) & (FC - 1))), SH = log2(32 / FC): the
// coalesced row-wise fill, the per-column reads and the transposes of all
// columns then each touch 32 distinct banks.  Smaller groups use a padded
// row stride of FC + 1.
template <int T, int FC>
struct ColTile {
    static constexpr bool swizzled = (T == 32) && FC > 1;
    static constexpr int ld = swizzled ? FC : FC + 1;
    static constexpr int sh = FC >= 32 ? 0 : (FC == 16 ? 1 : FC == 8 ? 2 : FC == 4 ? 3 : 4);
    static __device__ __forceinline__ int at(int y, int c)
    {
        if constexpr (swizzled)
            return y * FC + (c ^ ((y >> sh) & (FC - 1)));
        else
            return y * ld + c;
    }
    struct ColumnAddr {
        int c;
        __device__ __forceinline__ int operator()(int p) const { return at(p, c); }
    };
};

// Interleaved (float2) column tile for 32-lane groups and 8 columns: element
// (y, c) at y * 8 + (c ^ ((y >> 1) & 7)).  Sixteen consecutive rows of one
// column then fall in sixteen distinct 8-byte slots of a 128-byte window, so
// the per-column reads and both transpose phases (positions XOR-swizzled by
// tpos) are free of bank conflicts with 64-bit accesses.
struct ColTile2 {
    static __device__ __forceinline__ int at(int y, int c) { return y * 8 + (c ^ ((y >> 1) & 7)); }
    struct ColumnAddr {
        int c;
        __device__ __forceinline__ int operator()(int p) const { return at(p, c); }
    };
};

// float2 shared-memory access by 32-bit shared-window address.
__device__ __forceinline__ void sts2(uint32_t addr, float2 v)
{
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ float2 lds2(uint32_t addr)
{
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
    return v;
}

// Byte addresses in a ColTile2 tile that starts on a 2048-byte boundary.
// Slot (y, c) sits at byte 64 y + 8 (c ^ ((y >> 1) & 7)); for y = 32 a + u,
// u < 32, that is 2048 a + Q_c(u) with Q_c(u) = 64 u + 8 (c ^ ((u >> 1) & 7)).
// Q_c is XOR-linear: Q_c(t ^ k) = Q_c(t) ^ R(k), R(k) = 64 k + 8 ((k >> 1) & 7),
// so every transpose address of the 1024-point column transform is a lane
// constant XOR a compile-time constant (one logic instruction) plus an
// immediate offset.
__host__ __device__ constexpr uint32_t coltile_r(int k) { return 64u * k + 8u * ((k >> 1) & 7); }

// 1024-point transform of one tile column (the WarpFft<1024> four-step with
// T = E = 32): wbase = tile | Q_c(t) (transpose writes, element k1 at row
// 32 k1 + (t ^ k1)), rbase = (tile + 2048 t) | Q_c(t) (reads of row-block t).
template <int DIR>
__device__ __forceinline__ void col_fft_1024(float2 *v, const float2 *__restrict__ tw, uint32_t wbase,
                                             uint32_t rbase, int t)
{
    Dft<32, DIR>::run(v);
    WarpFft<1024>::twiddle<DIR>(v, tw, t);
#pragma unroll
    for (int k1 = 0; k1 < 32; k1++)
        sts2((wbase ^ coltile_r(k1)) + 2048u * k1, v[k1]);
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 32; j++)
        v[j] = lds2(rbase ^ coltile_r(j));
    __syncwarp();
    Dft<32, DIR>::run(v);
}

__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}

// Column pass for H <= 1024: CW warps per block, G = 32 / T columns per
// warp, FC = CW * G columns per block.  The FC-column tile is loaded into
// shared memory with coalesced accesses, each group transforms its column in
// registers using its own column of the tile as transpose buffer, and the tile
// is written back.  Spectrum in launch layout: block bx, register m, thread
// tid at spec[(bx * E + m) * (CW * 32) + tid].
template <int H, int CW>
__global__ void __launch_bounds__(CW * 32, FMVD_COL_MIN_BLOCKS) col_pass_w(const ColArgs a)
{
    using WF = WarpFft<H>;
    constexpr int T = WF::T, E = WF::E, G = 32 / T, FC = CW * G, NT = CW * 32;
    using TL = ColTile<T, FC>;
    extern __shared__ __align__(16) float smem[];
    float *tre = smem;
    float *tim = smem + H * TL::ld;
    const int W = a.W;
    const int p = blockIdx.y;
    const int x0 = blockIdx.x * FC;
    float2 *C = a.C + (size_t)p * H * W + x0;
    // this block's slice of the spectrum (contiguous in the launch layout)
    // is brought into L2 while the tile loads and the first transform runs
    pdl_launch_dependents();
    if (threadIdx.x == 0)
        bulk_prefetch_l2(a.spec + (size_t)blockIdx.x * E * NT, (uint32_t)(E * NT * sizeof(float2)));
    pdl_wait();

    if constexpr (T == 32 && FC == 8) {
        static_assert(H == 1024, "the interleaved tile path is the 1024-point column transform");
        // interleaved tile on a 2048-byte boundary, filled asynchronously
        const uint32_t s0 = smem_u32addr(smem);
        const uint32_t base = (s0 + 2047u) & ~2047u;
        float2 *tile = reinterpret_cast<float2 *>(reinterpret_cast<char *>(smem) + (base - s0));
#pragma unroll 8
        for (int u = threadIdx.x; u < H * 8; u += NT) {
            const int y = u >> 3, c = u & 7;
            cp_async8(tile + ColTile2::at(y, c), C + (size_t)y * W + c);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
        const int warp = threadIdx.x >> 5, t = threadIdx.x & 31;
        const uint32_t q = 64u * t + 8u * (warp ^ ((t >> 1) & 7));
        const uint32_t wbase = base | q, rbase = (base + 2048u * t) | q;
        float2 v[E];
#pragma unroll
        for (int m = 0; m < E; m++)
            v[m] = lds2(wbase + 2048u * m);  // row t + 32 m
        const float2 *sp = a.spec + (size_t)blockIdx.x * E * NT + threadIdx.x;
#pragma unroll 1
        for (int pass = 0; pass < 2; pass++) {
            col_fft_1024<-1>(v, a.tw, wbase, rbase, t);
            if (pass == 1)
                break;
#pragma unroll
            for (int m0 = 0; m0 < E; m0 += 8) {
                asm volatile("" ::: "memory");
#pragma unroll
                for (int m = m0; m < m0 + 8 && m < E; m++) {
                    const float2 z = cmul(v[m], __ldg(sp + (size_t)m * NT));
                    v[m] = make_float2(z.x, -z.y);
                }
            }
            asm volatile("" ::: "memory");
        }
#pragma unroll
        for (int m = 0; m < E; m++)
            sts2(wbase + 2048u * m, make_float2(v[m].x, -v[m].y));
        __syncthreads();
#pragma unroll 4
        for (int u = threadIdx.x; u < H * 4; u += NT) {
            const int y = u >> 2, c = 2 * (u & 3);
            const float2 e0 = tile[ColTile2::at(y, c)], e1 = tile[ColTile2::at(y, c + 1)];
            *reinterpret_cast<float4 *>(C + (size_t)y * W + c) = make_float4(e0.x, e0.y, e1.x, e1.y);
        }
        return;
    }

    constexpr int units = H * FC / 2;
#pragma unroll 4
    for (int u = threadIdx.x; u < units; u += NT) {
        const int c2 = u % (FC / 2), y = u / (FC / 2);
        const float4 q = *reinterpret_cast<const float4 *>(C + (size_t)y * W + 2 * c2);
        const int a0 = TL::at(y, 2 * c2), a1 = TL::at(y, 2 * c2 + 1);
        tre[a0] = q.x;
        tim[a0] = q.y;
        tre[a1] = q.z;
        tim[a1] = q.w;
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / T, t = lane % T;
    const typename TL::ColumnAddr addr{warp * G + g};
    float2 v[E];
#pragma unroll
    for (int m = 0; m < E; m++) {
        const int q = addr(t + T * m);
        v[m] = make_float2(tre[q], tim[q]);
    }
    // pass 0: forward transform, times the spectrum, conjugated; pass 1: the
    // same forward code gives the conjugate of the inverse transform
    const float2 *sp = a.spec + (size_t)blockIdx.x * E * NT + threadIdx.x;
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
        WF::template run_addr<-1>(v, a.tw, tre, tim, t, addr);
        if (pass == 1)
            break;
#pragma unroll
        for (int m0 = 0; m0 < E; m0 += 8) {
            asm volatile("" ::: "memory");
#pragma unroll
            for (int m = m0; m < m0 + 8 && m < E; m++) {
                const float2 z = cmul(v[m], __ldg(sp + (size_t)m * NT));
                v[m] = make_float2(z.x, -z.y);
            }
        }
        asm volatile("" ::: "memory");
    }
#pragma unroll
    for (int m = 0; m < E; m++) {
        const int q = addr(t + T * m);
        tre[q] = v[m].x;
        tim[q] = -v[m].y;
    }
    __syncthreads();
#pragma unroll 4
    for (int u = threadIdx.x; u < units; u += NT) {
        const int c2 = u % (FC / 2), y = u / (FC / 2);
        const int a0 = TL::at(y, 2 * c2), a1 = TL::at(y, 2 * c2 + 1);
        *reinterpret_cast<float4 *>(C + (size_t)y * W + 2 * c2) = make_float4(tre[a0], tim[a0], tre[a1], tim[a1]);
    }
}

// -------------------------------------- lines above 1024: R x 512 engine
// A line of N = R * kLineM points (R = 3..8, every supported length above
// 1024) is split over R groups of 16 lanes (half-warps), each running the
// 512-point warp FFT on one sub-line.  Frequencies R k1 + r live in sub-line
// r at position k1 (the work planes keep rows in this order between passes,
// and the column pass's spectrum follows it); space positions n1 + 512 q
// live in group q:
//   frequency -> space:  Z_r = FFT512(sub-line r), Z_r[n1] *= w_N^(r n1),
//                        x[n1 + 512 q] = sum_r Z_r[n1] w_R^(q r)
//   space -> frequency:  u_r[n1] = sum_q x[n1 + 512 q] w_R^(q r),
//                        u_r[n1] *= w_N^(r n1), sub-line r = FFT512(u_r)
// (forward sign; the inverse is conj(forward(conj))).  The sums over the R
// groups go through shared memory between two block barriers.

// v[m] *= w_N^(r n1), n1 = t + 16 m (twN: w_N^n, n < N): the table value
// for every eighth m, times powers of w_N^(16 r) in between (at most seven
// rounding steps; few table addresses live at once)
__device__ __forceinline__ void line_twiddle(float2 *v, const float2 *__restrict__ twN, int r, int t)
{
    const float2 step = __ldg(twN + 16 * r);
#pragma unroll
    for (int m0 = 0; m0 < 32; m0 += 8) {
        float2 w = __ldg(twN + r * (t + 16 * m0));
#pragma unroll
        for (int m = m0; m < m0 + 8; m++) {
            v[m] = cmul(v[m], w);
            if (m + 1 < m0 + 8)
                w = cmul(w, step);
        }
    }
}

// w_R^(r j) (twN: w_N^n with N = R * kLineM)
template <int R>
__device__ __forceinline__ float2 line_coefficient(const float2 *__restrict__ twN, int r, int j)
{
    return __ldg(twN + ((r * j) % R) * kLineM);
}

// Row pass for W = R * 512: R warps, two rows per block (half-warp h of warp
// r is group r of row h).
// SMEM: the launch bulk-copies each row's weight row (update) or data rows
// (divide) into shared memory after the buffers.
// DSTEP: the radix-R step as R-point DFTs per position (true) or as each
// group's weighted sum over all R sub-lines (false); the two schedules give
// the same transform with different instruction mixes (autotuner knob).
template <int R, int MODE, int BITS, bool NOOUT, bool SMEM, bool DSTEP>
__global__ void __launch_bounds__(R * 32, 16 / R) row_pass_r(const RowArgs a)
{
    using WF = WarpFft<kLineM>;
    constexpr int T = WF::T, E = WF::E, PF2 = WF::padded_f2, N = R * kLineM;
    static_assert(T == 16 && E == 32, "sub-lines are 512-point half-warp transforms");
    extern __shared__ __align__(16) float smem[];
    const int r = threadIdx.x >> 5;
    const int h = (threadIdx.x >> 4) & 1;
    const int t = threadIdx.x & 15;
    float2 *const lbuf = reinterpret_cast<float2 *>(smem) + (size_t)h * R * PF2;  // the row's R buffers
    float2 *const buf = lbuf + (size_t)r * PF2;
    const int y = blockIdx.x * 2 + h;
    const int p = blockIdx.y;
    float2 *row = a.b.C + ((size_t)p * a.d.H + y) * N + r * kLineM;
    RowWork<MODE, BITS, NOOUT, SMEM, false> work(a, p, y);

    // operand rows staged by bulk copies, issued now by one thread per row
    // (the weight row, a plan constant, before the dependency wait)
    constexpr bool staged = SMEM && MODE != ROW_INIT;
    __shared__ __align__(8) uint64_t sbar[2];
    const uint32_t rb = a.d.dataW * (MODE == ROW_UPDATE ? (uint32_t)sizeof(float) : (BITS == 8 ? 1u : 2u));
    const uint32_t rs = (rb + 15) & ~15u;
    char *const st = reinterpret_cast<char *>(smem) + sizeof(float2) * 2 * R * PF2 +
                     (size_t)h * (MODE == ROW_UPDATE ? rs : 2 * rs);
    pdl_launch_dependents();
    if (staged && threadIdx.x == 16 * h) {
        mbar_init(&sbar[h], 1);
        mbar_fence_init();
        if (MODE == ROW_UPDATE) {
            mbar_arrive_expect_tx(&sbar[h], rb);
            bulk_load(st, work.wrow, rb, &sbar[h]);
        }
    }
    pdl_wait();
    if (staged && MODE == ROW_DIVIDE && threadIdx.x == 16 * h) {
        mbar_arrive_expect_tx(&sbar[h], work.has1 ? 2 * rb : rb);
        bulk_load(st, work.src0, rb, &sbar[h]);
        if (work.has1)
            bulk_load(st + rs, work.src1, rb, &sbar[h]);
    }

    // the radix-R step across the row's R groups, v[m] <- sum_j (group j's
    // v[m]) w_R^(r j): every group puts its sub-line in its buffer (position
    // n1), then each half-warp of the row takes blocks of 16 positions n1
    // (block b = r, r + R, ...) and runs the R-point DFT over the R buffers
    // in place, and every group reads its own buffer back
    const auto line_dft = [&](float2 *v) {
#pragma unroll
        for (int m = 0; m < E; m++)
            buf[t + T * m] = v[m];
        __syncthreads();
        if constexpr (!DSTEP) {
            // each group sums all R sub-lines at its own positions
#pragma unroll
            for (int m = 0; m < E; m++)
                v[m] = lbuf[t + T * m];
#pragma unroll
            for (int j = 1; j < R; j++) {
                const float2 cj = line_coefficient<R>(a.twN, r, j);
#pragma unroll
                for (int m = 0; m < E; m++)
                    v[m] = cadd(v[m], cmul(lbuf[j * PF2 + t + T * m], cj));
            }
            __syncthreads();
        } else {
#pragma unroll 1
            for (int b = r; b < kLineM / 16; b += R) {
                float2 z[R];
#pragma unroll
                for (int q = 0; q < R; q++)
                    z[q] = lbuf[q * PF2 + 16 * b + t];
                SmallDft<R>::run(z);
#pragma unroll
                for (int q = 0; q < R; q++)
                    lbuf[q * PF2 + 16 * b + t] = z[q];
            }
            __syncthreads();
#pragma unroll
            for (int m = 0; m < E; m++)
                v[m] = buf[t + T * m];
        }
    };

    // pass 0: frequency -> space (the inverse as conj(forward(conj))) and
    // the element-wise step; pass 1: space -> frequency.  The rolled loop
    // keeps one copy of the 512-point transform.
    float2 v[E];
    if (MODE == ROW_INIT) {
#pragma unroll
        for (int m = 0; m < E; m++) {
            v[m] = make_float2(0.f, 0.f);
            work.apply(r * kLineM + t + T * m, v[m]);
        }
    } else {
#pragma unroll
        for (int m = 0; m < E; m++) {
            const float2 x = row[t + T * m];
            v[m] = make_float2(x.x, -x.y);
        }
    }
#pragma unroll 1
    for (int pass = MODE == ROW_INIT ? 1 : 0; pass < 2; pass++) {
        if (pass == 1) {
            line_dft(v);
            line_twiddle(v, a.twN, r, t);
        }
        WF::template run_padded<-1>(v, a.tw, buf, t);
        if (pass == 1)
            break;
        // the operand rows of this group's space block (positions r * 512 ..
        // r * 512 + 511) are requested into L1 here and read after the sum
        if (MODE == ROW_UPDATE) {
            prefetch_l1(work.est + r * kLineM + 16 * t);
            prefetch_l1(work.est + r * kLineM + 16 * (t + 16));
            if (!staged)
                prefetch_l1(work.wrow + clamp_src(r * kLineM + 32 * t, a.d.dataW, a.d.bxW));
        } else if (MODE == ROW_DIVIDE && !staged) {
            const int sx = clamp_src(r * kLineM + 64 * (t & 7), a.d.dataW, a.d.bxD);
            prefetch_l1((const char *)(t < 8 ? work.src0 : work.src1) + (size_t)sx * (BITS == 8 ? 1 : 2));
        }
        line_twiddle(v, a.twN, r, t);
        line_dft(v);
        if (staged) {
            if (!mbar_wait(&sbar[h], 0)) {
                // the copy did not land in time: flag it (the host reports the
                // batch as failed) and wait once more so no copy is left in flight
                if (threadIdx.x == 16 * h)
                    atomicExch(a.b.status, 1);
                mbar_wait(&sbar[h], 0);
            }
            if (MODE == ROW_UPDATE) {
                work.s_w = smem_u32addr(st);
            } else {
                work.s_src0 = smem_u32addr(st);
                work.s_src1 = work.has1 ? smem_u32addr(st + rs) : work.s_src0;
            }
        }
#pragma unroll
        for (int m = 0; m < E; m++) {
            v[m].y = -v[m].y;
            work.apply(r * kLineM + t + T * m, v[m]);
        }
        if (MODE == ROW_UPDATE && !NOOUT && a.last)
            return;
    }
#pragma unroll
    for (int m = 0; m < E; m++)
        row[t + T * m] = v[m];
}

// Column tile of the line engine: two columns, element (y, c) at float2
// 2 y + (c ^ ((y >> 3) & 1)): sixteen consecutive rows of one column fall in
// sixteen distinct 8-byte slots of a 256-byte window.  With the tile on a
// 256-byte boundary, row y = 512 r + 16 a + u (u < 16) of column c is at
// byte 8192 r + 256 a + 8 Q_c(u), Q_c(u) = 2 u + (c ^ ((u >> 3) & 1)), and
// Q_c is XOR-linear: Q_c(t ^ k) = Q_c(t) ^ R16(k), R16(k) = 2 k + ((k >> 3) & 1).
__device__ __forceinline__ int coltile_r(int y, int c) { return 2 * y + (c ^ ((y >> 3) & 1)); }
__host__ __device__ constexpr uint32_t coltile16_r(int k) { return 2u * k + ((k >> 3) & 1); }

// 512-point transform (WarpFft<512>: T = 16, E = 32) of one sub-line of a
// line-engine column tile, its own rows as transpose space:
// wbase = sub-line start | 8 Q_c(t), rbase = (sub-line start + 256 t) | 8 Q_c(t).
template <int DIR, typename TW>
__device__ __forceinline__ void col_fft_512(float2 *v, const TW &tw, uint32_t wbase, uint32_t rbase, int t)
{
    using WF = WarpFft<kLineM>;
    Dft<32, DIR>::run(v);
    WF::template twiddle<DIR>(v, tw, t);
#pragma unroll
    for (int k1 = 0; k1 < 32; k1++)
        sts2((wbase ^ (8u * coltile16_r(k1 & 15))) + 256u * k1, v[k1]);
    __syncwarp();
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int j = 0; j < 16; j++)
            v[s * 16 + j] = lds2((rbase ^ (8u * coltile16_r(j))) + 4096u * s);
    __syncwarp();
    Dft<16, DIR>::run(v);
    Dft<16, DIR>::run(v + 16);
    WF::reorder(v);
}

// Column pass for H = R * 512: R warps, two columns per block (half-warp cc
// of warp r is group r of column cc).  Spectrum in launch layout: block bx,
// register m, thread tid at spec[(bx * 32 + m) * (32 R) + tid].  Resident
// blocks per SM: 16 / R, except 4 (not 5) for R = 3, where the register cap of
// five blocks spills and four run 2 % faster.
template <int R>
constexpr int col_r_blocks() { return R == 3 ? 4 : 16 / R; }

template <int R, bool DSTEP>
__global__ void __launch_bounds__(R * 32, col_r_blocks<R>()) col_pass_r(const ColArgs a)
{
    using WF = WarpFft<kLineM>;
    static_assert(WF::T == 16 && WF::E == 32, "sub-lines are 512-point half-warp transforms");
    constexpr int E = WF::E, H = R * kLineM, NT = R * 32;
    extern __shared__ __align__(16) float smem[];
    const uint32_t s0 = smem_u32addr(smem);
    const uint32_t base = (s0 + 255u) & ~255u;
    float2 *tile = reinterpret_cast<float2 *>(reinterpret_cast<char *>(smem) + (base - s0));
    const int W = a.W;
    const int p = blockIdx.y;
    float2 *C = a.C + (size_t)p * H * W + 2 * blockIdx.x;
    // this block's slice of the spectrum (contiguous in the launch layout)
    // is brought into L2 while the tile loads and the first transform runs
    pdl_launch_dependents();
    if (threadIdx.x == 0)
        bulk_prefetch_l2(a.spec + (size_t)blockIdx.x * E * NT, (uint32_t)(E * NT * sizeof(float2)));
    pdl_wait();
#pragma unroll 8
    for (int i = 0; i < 2 * H / NT; i++) {
        const int u = threadIdx.x + i * NT;
        const int y = u >> 1, c = u & 1;
        cp_async8(tile + coltile_r(y, c), C + (size_t)y * W + c);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    const int r = threadIdx.x >> 5;
    const int cc = (threadIdx.x >> 4) & 1;
    const int t = threadIdx.x & 15;
    const uint32_t q = 8u * (2 * t + (cc ^ ((t >> 3) & 1)));
    const uint32_t col = base + q;                  // + 8192 j + 256 m: row 512 j + t + 16 m
    const uint32_t seg = base + 8192u * r;          // this group's sub-line
    const uint32_t wbase = seg | q, rbase = (seg + 256u * t) | q;

    // The radix-R step of both columns in place in the tile: each half-warp
    // takes blocks of 16 positions n1 of its column (block b = r, r + R, ...)
    // and runs the R-point DFT over the rows 512 q + n1 (q < R); with CONJ the
    // results are stored conjugated.  The tile address of row 512 q + 16 b + t
    // of this column is col + 8192 q + 256 b.
    const auto column_dft = [&](auto conj_out) {
#pragma unroll 1
        for (int b = r; b < kLineM / 16; b += R) {
            float2 z[R];
#pragma unroll
            for (int q = 0; q < R; q++)
                z[q] = lds2(col + 8192u * q + 256u * b);
            SmallDft<R>::run(z);
#pragma unroll
            for (int q = 0; q < R; q++)
                sts2(col + 8192u * q + 256u * b, decltype(conj_out)::value ? make_float2(z[q].x, -z[q].y) : z[q]);
        }
    };

    // the other schedule: v[m] = sum_j (row 512 j + t + 16 m of this column) w_R^(r j)
    const auto column_sum = [&](float2 *v) {
#pragma unroll
        for (int m = 0; m < E; m++)
            v[m] = lds2(col + 256u * m);
#pragma unroll
        for (int j = 1; j < R; j++) {
            const float2 cj = line_coefficient<R>(a.twN, r, j);
#pragma unroll
            for (int m0 = 0; m0 < E; m0 += 8) {
                asm volatile("" ::: "memory");  // bounds the loads in flight
#pragma unroll
                for (int m = m0; m < m0 + 8; m++)
                    v[m] = cadd(v[m], cmul(lds2(col + 8192u * j + 256u * m), cj));
            }
        }
        asm volatile("" ::: "memory");
    };

    float2 v[E];
    // pass 0: space -> frequency, times the spectrum, conjugated; pass 1:
    // the same forward pipeline then runs frequency -> space.  The rolled
    // loop keeps one copy of the transform (its table loads are not kept
    // live from one copy to the next).
    const float2 *sp = a.spec + (size_t)blockIdx.x * E * NT + threadIdx.x;
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 0) {
            if constexpr (DSTEP) {
                column_dft(std::false_type());
                __syncthreads();  // every block of positions has its radix-R step
#pragma unroll
                for (int m = 0; m < E; m++)
                    v[m] = lds2(col + 8192u * r + 256u * m);  // row 512 r + t + 16 m: this group's sub-line
                __syncwarp();  // read before this warp's transposes overwrite its segment
            } else {
                column_sum(v);
                __syncthreads();  // every group has read the column before transposes overwrite it
            }
            line_twiddle(v, a.twN, r, t);
        }
        col_fft_512<-1>(v, a.tw, wbase, rbase, t);
        if (pass == 1)
            break;
#pragma unroll
        for (int m0 = 0; m0 < E; m0 += 8) {
            asm volatile("" ::: "memory");
#pragma unroll
            for (int m = m0; m < m0 + 8; m++) {
                const float2 z = cmul(v[m], __ldg(sp + (size_t)m * NT));
                v[m] = make_float2(z.x, -z.y);
            }
        }
        asm volatile("" ::: "memory");
    }
    line_twiddle(v, a.twN, r, t);
#pragma unroll
    for (int m = 0; m < E; m++)
        sts2(seg + q + 256u * m, v[m]);  // row 512 r + t + 16 m
    __syncthreads();
    if constexpr (DSTEP) {
        column_dft(std::true_type());
    } else {
        column_sum(v);
        __syncthreads();
#pragma unroll
        for (int m = 0; m < E; m++)
            sts2(seg + q + 256u * m, make_float2(v[m].x, -v[m].y));
    }
    __syncthreads();
    // row y's two elements are the 16 bytes at 16 y, column 1 first where
    // bit 3 of y is set: one 16-byte load per row
#pragma unroll 4
    for (int i = 0; i < H / NT; i++) {
        const int y = threadIdx.x + i * NT;
        const float4 e = reinterpret_cast<const float4 *>(tile)[y];
        *reinterpret_cast<float4 *>(C + (size_t)y * W) =
            (y >> 3) & 1 ? make_float4(e.z, e.w, e.x, e.y) : e;
    }
}

// Frequency of stored column (or row position) j of a line of length n:
// natural up to 1024, the R x 512 order above.
__host__ __device__ __forceinline__ int stored_frequency(int j, int n)
{
    if (n <= 1024)
        return j;
    const int R = n / kLineM;
    return R * (j % kLineM) + j / kLineM;
}

// Launch layout of the line engine's column-pass spectrum: block bx
// (stored columns 2 bx, 2 bx + 1), register m, thread tid = 32 r + 16 cc + t
// holds frequency ky = R (t + 16 m) + r of stored column 2 bx + cc.
__global__ void permute_spectrum_r(const float2 *__restrict__ nat, float2 *__restrict__ out, int H, int W, float scale)
{
    const int R = H / kLineM, NT = 32 * R;
    const size_t total = (size_t)H * W;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int tid = (int)(i % NT);
        const int m = (int)((i / NT) % 32);
        const int bx = (int)(i / ((size_t)NT * 32));
        const int r = tid >> 5, cc = (tid >> 4) & 1, t = tid & 15;
        const int ky = R * (t + 16 * m) + r;
        const int kx = stored_frequency(2 * bx + cc, W);
        const float2 k = nat[(size_t)ky * W + kx];
        out[i] = make_float2(k.x * scale, k.y * scale);
    }
}

// Launch layout of the column-pass spectrum for the warp engine.
__global__ void permute_spectrum_w(const float2 *__restrict__ nat, float2 *__restrict__ out, int H, int W, int T,
                                   int CW, float scale)
{
    const int E = H / T, G = 32 / T, FC = CW * G, NT = CW * 32;
    const size_t total = (size_t)H * W;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int tid = (int)(i % NT);
        const int m = (int)((i / NT) % E);
        const int bx = (int)(i / ((size_t)NT * E));
        const int warp = tid >> 5, lane = tid & 31;
        const int g = lane / T, t = lane % T;
        const int n = t + T * m;
        const int col = stored_frequency(bx * FC + warp * G + g, W);
        const float2 k = nat[(size_t)n * W + col];
        out[i] = make_float2(k.x * scale, k.y * scale);
    }
}

// Plan-time kernels in FP32 (the reference builds its kernel spectra with an
// FP32 cuFFT, fmvd_deconvolve.impl.cpp:66-76).  Sums use compensated
// (Kahan) accumulation with explicitly rounded operations, so that the
// spectra carry about FP32 rounding of the exact value whatever the kernel
// size.
struct KahanSum {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float v)
    {
        const float y = __fsub_rn(v, c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
};

// Separable direct DFT of a small kernel placed at (y - kH/2, x - kW/2) mod (H, W).
// Step 1: A[y][v] = sum_x k[y][x] exp(-2 pi i v (x - cx) / W)
__global__ void kspec_rows(const float *__restrict__ k, int kH, int kW, int W, const float2 *__restrict__ twW,
                           float2 *__restrict__ A)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (v >= W)
        return;
    KahanSum re, im;
    const int cx = kW / 2;
    for (int x = 0; x < kW; x++) {
        const long long ph = ((long long)v * (x - cx)) % W;
        const float2 t = twW[ph < 0 ? ph + W : ph];
        const float kv = k[y * kW + x];
        re.add(__fmul_rn(kv, t.x));
        im.add(__fmul_rn(kv, t.y));
    }
    A[(size_t)y * W + v] = make_float2(re.s, im.s);
}

// Step 2: K[u][v] = sum_y A[y][v] exp(-2 pi i u (y - cy) / H)
__global__ void kspec_cols(const float2 *__restrict__ A, int kH, int H, int W, const float2 *__restrict__ twH,
                           float2 *__restrict__ K)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int u = blockIdx.y;
    if (v >= W)
        return;
    KahanSum re, im;
    const int cy = kH / 2;
    for (int y = 0; y < kH; y++) {
        const long long ph = ((long long)u * (y - cy)) % H;
        const float2 t = twH[ph < 0 ? ph + H : ph];
        const float2 a = A[(size_t)y * W + v];
        re.add(__fmul_rn(a.x, t.x));
        re.add(-__fmul_rn(a.y, t.y));
        im.add(__fmul_rn(a.x, t.y));
        im.add(__fmul_rn(a.y, t.x));
    }
    K[(size_t)u * W + v] = make_float2(re.s, im.s);
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

__global__ void conv_same_kernel(const float *__restrict__ img, int dH, int dW, const float *__restrict__ k, int kH,
                                 int kW, int fH, int fW, float *__restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= dW || y >= dH)
        return;
    KahanSum acc;
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
            acc.add(__fmul_rn(img[(size_t)sy * dW + sx], k[ky * kW + kx]));
        }
    }
    out[(size_t)y * dW + x] = acc.s;
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


// Warps per column block of the warp engine: the largest of 8, 4, 2 whose
// columns per block divide W.
static int col_warps(int H, int W)
{
    const int G = 32 / warp_fft_lanes(H);
    for (int cw = FMVD_COL_MAX_WARPS; cw > 1; cw /= 2)
        if (W % (cw * G) == 0)
            return cw;
    return 1;
}

int rl_col_warps(int H, int W, int requested)
{
    if (H > 1024)
        return 0;  // line engine: fixed two-column tile
    if (requested == 0)
        return col_warps(H, W);
    const int G = 32 / warp_fft_lanes(H);
    const bool ok = (requested == 2 || requested == 4 || requested == 8) && requested <= FMVD_COL_MAX_WARPS &&
                    W % (requested * G) == 0;
    return ok ? requested : -1;
}

size_t rl_spectrum_elems(int H, int W) { return (size_t)H * W; }

// Launch of an RL pass with programmatic dependent launch on stream s (the
// pass's blocks may start while the previous kernel of the stream finishes;
// the pass waits for it before reading its results).  Falls back to a plain
// launch if the attribute is refused.
template <typename A>
static void launch_pass(void (*kern)(const A), dim3 grid, dim3 block, size_t smem, cudaStream_t s, const A &args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, kern, args) != cudaSuccess) {
        cudaGetLastError();  // clear the refusal; launch without the attribute
        kern<<<grid, block, smem, s>>>(args);
    }
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

static bool aligned16(const void *p, size_t bytes) { return ((uintptr_t)p % 16 == 0) && bytes % 16 == 0; }

// Warp row-pass variant for a launch (update passes: noout when not the
// last view; sm when the operand rows are bulk-copied into shared memory).
template <int W, int MODE, int BITS>
static void pick_row_w(bool noout, bool sm, void (*&kern)(const RowArgs), unsigned *&m)
{
    static unsigned mask[4] = {0, 0, 0, 0};
    constexpr bool U = MODE == ROW_UPDATE;
    if (noout)
        kern = sm ? row_pass_w<W, MODE, BITS, U, true> : row_pass_w<W, MODE, BITS, U, false>;
    else
        kern = sm ? row_pass_w<W, MODE, BITS, false, true> : row_pass_w<W, MODE, BITS, false, false>;
    m = &mask[(noout ? 1 : 0) + (sm ? 2 : 0)];
}

// Line-engine row-pass variant for a launch (per sample width; update
// passes per last / not last).
template <int R, int MODE, int BITS, bool DSTEP>
static void pick_row_r_bits(bool noout, bool sm, void (*&kern)(const RowArgs), unsigned *&m)
{
    static unsigned mask[4] = {0, 0, 0, 0};
    constexpr bool U = MODE == ROW_UPDATE;
    if (noout)
        kern = sm ? row_pass_r<R, MODE, BITS, U, true, DSTEP> : row_pass_r<R, MODE, BITS, U, false, DSTEP>;
    else
        kern = sm ? row_pass_r<R, MODE, BITS, false, true, DSTEP> : row_pass_r<R, MODE, BITS, false, false, DSTEP>;
    m = &mask[(noout ? 1 : 0) + (sm ? 2 : 0)];
}

// (sm: the operand rows may be bulk-copied into shared memory)
template <int R, int MODE, bool DSTEP>
static void pick_row_r(const RowArgs &a, bool sm, void (*&kern)(const RowArgs), unsigned *&m)
{
    static unsigned mask0 = 0;
    const bool noout = MODE == ROW_UPDATE && !a.last;
    if constexpr (MODE == ROW_INIT) {
        kern = row_pass_r<R, MODE, 0, false, false, DSTEP>;
        m = &mask0;
    } else if (a.d.bits == 16) {
        pick_row_r_bits<R, MODE, 16, DSTEP>(noout, sm, kern, m);
    } else {
        pick_row_r_bits<R, MODE, 8, DSTEP>(noout, sm, kern, m);
    }
}

template <int W, int MODE>
static void launch_row(const RowArgs &a0, cudaStream_t s)
{
    if constexpr (W <= 1024) {
        using WF = WarpFft<W>;
        constexpr int G = 32 / WF::T;
        RowArgs a = a0;
        const size_t es = a.d.bits == 16 ? 2 : 1;
        a.bulk_data = aligned16(a.b.data, a.d.dataW * es) && (a.b.view_stride * es) % 16 == 0 &&
                      (a.b.plane_stride * es) % 16 == 0;
        a.bulk_weights = aligned16(a.b.weights, a.d.dataW * sizeof(float)) &&
                         ((size_t)a.d.dataH * a.d.dataW * sizeof(float)) % 16 == 0;
        size_t pf = 0;
        if (MODE == ROW_UPDATE)
            pf = a.bulk_weights ? a.d.dataW * sizeof(float) : 0;
        else if (MODE == ROW_DIVIDE && a.bulk_data)
            pf = 2 * ((a.d.dataW * es + 15) & ~(size_t)15);
        static_assert(WF::padded_f2 >= W, "the update pass lands the estimate row in the transpose buffer");
        a.group_floats = WF::padded_floats + (int)(pf / sizeof(float));
        const size_t smem = sizeof(float) * kRowWarps * G * (size_t)a.group_floats;
        // the element-wise step is compiled for the sample width
        // compiled per sample width, per operand rows in shared memory or
        // not, and for the update pass per last / not last
        void (*kern)(const RowArgs);
        unsigned *m;
        const bool noout = MODE == ROW_UPDATE && !a.last;
        const bool sm = MODE == ROW_UPDATE ? a.bulk_weights != 0 : (MODE == ROW_DIVIDE && a.bulk_data != 0);
        if constexpr (MODE == ROW_INIT) {
            static unsigned mask0 = 0;
            kern = row_pass_w<W, MODE, 0, false, false>;
            m = &mask0;
        } else if (a.d.bits == 16) {
            pick_row_w<W, MODE, 16>(noout, sm, kern, m);
        } else {
            pick_row_w<W, MODE, 8>(noout, sm, kern, m);
        }
        configure_smem(kern, 200 * 1024, *m);
        dim3 grid((a.d.H + kRowWarps * G - 1) / (kRowWarps * G), a.b.npairs);
        launch_pass(kern, grid, dim3(kRowWarps * 32), smem, s, a);
    } else {
        constexpr int R = W / kLineM;
        static_assert(W % kLineM == 0 && R >= 3 && R <= 8, "rows above 1024 are 3..8 sub-lines of 512");
        RowArgs a = a0;
        const size_t es = a.d.bits == 16 ? 2 : 1;
        a.bulk_data = aligned16(a.b.data, a.d.dataW * es) && (a.b.view_stride * es) % 16 == 0 &&
                      (a.b.plane_stride * es) % 16 == 0;
        a.bulk_weights = aligned16(a.b.weights, a.d.dataW * sizeof(float)) &&
                         ((size_t)a.d.dataH * a.d.dataW * sizeof(float)) % 16 == 0;
        const bool sm = MODE == ROW_UPDATE ? a.bulk_weights != 0 : (MODE == ROW_DIVIDE && a.bulk_data != 0);
        size_t smem = sizeof(float2) * 2 * R * WarpFft<kLineM>::padded_f2;
        if (sm) {
            const size_t rs = ((size_t)a.d.dataW * (MODE == ROW_UPDATE ? sizeof(float) : es) + 15) & ~(size_t)15;
            smem += 2 * (MODE == ROW_UPDATE ? rs : 2 * rs);
        }
        void (*kern)(const RowArgs);
        unsigned *m;
        if (a.d.radix_step == kRadixSums)
            pick_row_r<R, MODE, false>(a, sm, kern, m);
        else
            pick_row_r<R, MODE, true>(a, sm, kern, m);
        configure_smem(kern, 200 * 1024, *m);
        dim3 grid(a.d.H / 2, a.b.npairs);
        launch_pass(kern, grid, dim3(R * 32), smem, s, a);
    }
    g_launches++;
}

template <int H, int CW>
static void launch_col_w(const ColArgs &a, int npairs, cudaStream_t s)
{
    using WF = WarpFft<H>;
    constexpr int FC = CW * (32 / WF::T);
    // the interleaved-tile path (T = 32, 8 columns) aligns its tile to 2048 bytes
    constexpr size_t smem = sizeof(float) * 2 * H * ColTile<WF::T, FC>::ld + (WF::T == 32 && FC == 8 ? 2048 : 0);
    auto kern = col_pass_w<H, CW>;
    static unsigned mask = 0;
    configure_smem(kern, smem, mask);
    dim3 grid(a.W / FC, npairs);
    launch_pass(kern, grid, dim3(CW * 32), smem, s, a);
}

template <int H>
static void launch_col(const ColArgs &a, int npairs, int cw, int radix_step, cudaStream_t s)
{
    if constexpr (H <= 1024) {
        switch (cw) {
        case 8: launch_col_w<H, 8>(a, npairs, s); break;
        case 4: launch_col_w<H, 4>(a, npairs, s); break;
        default: launch_col_w<H, 2>(a, npairs, s); break;
        }
    } else {
        constexpr int R = H / kLineM;
        static_assert(H % kLineM == 0 && R >= 3 && R <= 8, "columns above 1024 are 3..8 sub-lines of 512");
        constexpr size_t smem = sizeof(float2) * 2 * H + 256;  // tile aligned to 256 bytes in the kernel
        const bool sums = radix_step == kRadixSums;
        auto kern = sums ? col_pass_r<R, false> : col_pass_r<R, true>;
        static unsigned mask[2] = {0, 0};
        configure_smem(kern, smem, mask[sums ? 1 : 0]);
        dim3 grid(a.W / 2, npairs);
        launch_pass(kern, grid, dim3(R * 32), smem, s, a);
    }
    g_launches++;
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
    RowArgs a{d, b, t.wtwW, 0, 0, 0, 0, 0, t.twW};
    dispatch_row<ROW_INIT>(a, s);
}

void rl_divide(const RlDims &d, const RlBatch &b, const RlTables &t, int view, cudaStream_t s)
{
    RowArgs a{d, b, t.wtwW, view, 0, 0, 0, 0, t.twW};
    dispatch_row<ROW_DIVIDE>(a, s);
}

void rl_update(const RlDims &d, const RlBatch &b, const RlTables &t, int view, bool last, cudaStream_t s)
{
    RowArgs a{d, b, t.wtwW, view, last ? 1 : 0, 0, 0, 0, t.twW};
    dispatch_row<ROW_UPDATE>(a, s);
}

void rl_col(const RlDims &d, const RlBatch &b, const RlTables &t, const float2 *spectrum, cudaStream_t s)
{
    ColArgs a{b.C, spectrum, t.wtwH, d.H, d.W, t.twH};
    switch (d.H) {
#define X(N) \
    case N: launch_col<N>(a, b.npairs, d.col_warps ? d.col_warps : col_warps(d.H, d.W), d.radix_step, s); break;
        FMVD_FOR_EACH_LENGTH(X)
#undef X
    default: break;
    }
}

int rl_warp_lanes(int n) { return n <= 1024 ? warp_fft_lanes(n) : 0; }

int rl_warp_twiddle_entries(int n)
{
    if (n > 1024)
        return rl_warp_twiddle_entries(kLineM);
    const int T = rl_warp_lanes(n);
    if (T == 0)
        return n;
    const int E = n / T, R = E < kWarpTwiddleRun ? E : kWarpTwiddleRun;
    const int used = (E / R + 1) * T;
    return used > n ? used : n;
}

void rl_kernel_spectrum(const float *d_kernel, int kH, int kW, int H, int W, const float2 *twH, const float2 *twW,
                        float2 *work, float2 *d_out, int cw, cudaStream_t s)
{
    float2 *A = work;
    float2 *K = work + (size_t)kH * W;
    kspec_rows<<<dim3((W + 127) / 128, kH), 128, 0, s>>>(d_kernel, kH, kW, W, twW, A);
    kspec_cols<<<dim3((W + 127) / 128, H), 128, 0, s>>>(A, kH, H, W, twH, K);
    const size_t total = rl_spectrum_elems(H, W);
    const int blocks = (int)((total + 255) / 256 > 4096 ? 4096 : (total + 255) / 256);
    // 1 / (H W), rounded once to float (the reference's modulateAndNormalize
    // factor, fmvd_deconvolve_cuda.cu:369)
    const float scale = (float)(1.0 / ((double)H * (double)W));
    if (H <= 1024) {
        permute_spectrum_w<<<blocks, 256, 0, s>>>(K, d_out, H, W, warp_fft_lanes(H), cw ? cw : col_warps(H, W),
                                                  scale);
    } else {
        permute_spectrum_r<<<blocks, 256, 0, s>>>(K, d_out, H, W, scale);
    }
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

void rl_conv_same(const float *d_img, int dH, int dW, const float *d_k, int kH, int kW, float *d_out, cudaStream_t s)
{
    const int fH = snap_transform_size(dH + kH - 1);
    const int fW = snap_transform_size(dW + kW - 1);
    conv_same_kernel<<<dim3((dW + 127) / 128, dH), 128, 0, s>>>(d_img, dH, dW, d_k, kH, kW, fH, fW, d_out);
}

} // namespace fmvd
