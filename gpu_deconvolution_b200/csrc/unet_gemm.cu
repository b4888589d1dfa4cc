// BF16 implicit-GEMM 3x3 / 1x1 convolutions on the tcgen05 tensor cores
// (FP32 accumulation in tensor memory), for the warm-start network.
//
// Activations are NHWC bf16; weights [Cout][taps][Cin] bf16.  Two GEMM forms:
//
//   mode 0 (forward and data gradient): D[pixel][co] = sum over taps t and
//     input channels ci of A[pixel + off(t)][ci] * B[co][t][ci].  A tile is
//     128 output pixels (a bw x bh patch of one image); each K block is one
//     tap and CB input channels, loaded by a 4-D TMA box whose out-of-image
//     part arrives as zeros (the convolution's zero padding).  Both operands
//     are K-major.  The epilogue adds the bias and an optional skip tensor,
//     applies ReLU, zeroes where a mask tensor is <= 0 (the ReLU derivative
//     of the data gradient) and stores bf16 (and/or fp32).
//   mode 1 (weight gradient): D[co][ci] = sum over pixels p of
//     G[p][co] * X[p + off(t)][ci] for one tap t.  K runs over pixels, so
//     both operands are MN-major (channels contiguous); the pixel range is
//     split over CTAs and the FP32 partial sums are added into dW with
//     atomics.
//
// One CTA of 4 warps computes a 128 x BN tile: warp 0 lane 0 issues the TMA
// loads into a ring of shared-memory stages, warp 1 lane 0 issues the MMAs
// and commits each stage back to the producer, then all warps read the
// accumulator from tensor memory.  Every mbarrier wait is bounded: on a
// timeout the CTA records an error in *status and finishes without hanging.
#include "fmvd_internal.h"
#include "tma_util.cuh"
#include "umma.cuh"
#include "unet.h"

#include <cuda_bf16.h>
#include <stdio.h>

namespace fmvd {
namespace unet {

using bf16 = __nv_bfloat16;
constexpr int kKP = 64;  // pixels per K block of the weight gradient

__host__ __device__ constexpr uint32_t align1k(uint32_t b) { return (b + 1023u) & ~1023u; }

template <int MODE, int CBA, int CBB, int BN>
struct GemmCfg {
    static constexpr int RA = CBA * 2, RB = CBB * 2;  // bytes per staged row
    static constexpr uint32_t SA = MODE == 0 ? 128u * RA : (uint32_t)kKP * 128u * 2u;
    static constexpr uint32_t SB = MODE == 0 ? (uint32_t)BN * RB : (uint32_t)kKP * BN * 2u;
    static constexpr uint32_t SA_AL = align1k(SA), SB_AL = align1k(SB);
    static constexpr uint32_t STAGE = SA_AL + SB_AL;
    static constexpr int STAGES = 98304u / STAGE >= 4 ? 4 : (98304u / STAGE >= 2 ? (int)(98304u / STAGE) : 2);
    static constexpr uint32_t SMEM = STAGES * STAGE + 1024;
    static constexpr int TCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    static constexpr int KSTEPS = MODE == 0 ? CBA / 16 : kKP / 16;
    static_assert(MODE == 1 || CBA == CBB, "forward K blocks share one channel block");
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "N tile");
};

__device__ __forceinline__ void tap_offset(int taps, int t, int &dy, int &dx)
{
    if (taps == 9) {
        dy = t / 3 - 1;
        dx = t % 3 - 1;
    } else {
        dy = dx = 0;
    }
}

template <int MODE, int CBA, int CBB, int BN>
__global__ void __launch_bounds__(128, 1)
    conv_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const GemmArgs g)
{
    using C = GemmCfg<MODE, CBA, CBB, BN>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *sa = smem;
    uint8_t *sb = smem + C::STAGES * C::SA_AL;
    __shared__ __align__(8) uint64_t full[C::STAGES], empty[C::STAGES], done;
    __shared__ uint32_t tmem_sh;
    __shared__ int fail_sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // ---- tile coordinates
    int n = 0, y0 = 0, x0 = 0, co0 = 0, ci0 = 0, tap = 0, kb0 = 0, nk = 0;
    if (MODE == 0) {
        const int tx = g.W / g.bw, ty = g.H / g.bh;
        const int tile = blockIdx.x;
        n = tile / (tx * ty);
        const int r = tile % (tx * ty);
        y0 = (r / tx) * g.bh;
        x0 = (r % tx) * g.bw;
        co0 = blockIdx.y * BN;
        nk = g.taps * (g.cin / CBA);
    } else {
        tap = blockIdx.x % g.taps;
        co0 = (blockIdx.x / g.taps) * 128;
        ci0 = blockIdx.z * BN;
        const int total = (int)(((long long)g.N * g.H * g.W) / kKP);
        kb0 = blockIdx.y * g.kchunk;
        nk = min(g.kchunk, total - kb0);
    }
    // weight-gradient A groups that hold output channels (the rest stay zero)
    const int ga_valid = MODE == 1 ? min(128 / CBA, (g.cout - co0 + CBA - 1) / CBA) : 0;

    if (MODE == 1 && ga_valid < 128 / CBA) {
        const int zero_from = ga_valid * kKP * C::RA;
        for (int s = 0; s < C::STAGES; s++)
            for (int i = zero_from / 16 + threadIdx.x; i < (int)(C::SA / 16); i += blockDim.x)
                reinterpret_cast<uint4 *>(sa + s * C::SA_AL)[i] = make_uint4(0, 0, 0, 0);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; s++) {
            umma::bar_init(&full[s], 1);
            umma::bar_init(&empty[s], 1);
        }
        umma::bar_init(&done, 1);
        umma::bar_fence_init();
        fail_sh = 0;
    }
    if (warp == 0) {
        umma::tmem_alloc(&tmem_sh, C::TCOLS);
        umma::tmem_relinquish();
    }
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
    const uint32_t tmem = tmem_sh;

    if (warp == 0 && lane == 0) {
        // ---- producer: TMA loads of the K blocks into the stage ring
        const uint32_t bytes = MODE == 0 ? C::SA + C::SB
                                         : (uint32_t)ga_valid * kKP * C::RA + (uint32_t)kKP * BN * 2u;
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb % C::STAGES, round = kb / C::STAGES;
            if (round > 0 && !umma::bar_wait(&empty[s], (round - 1) & 1)) {
                fail_sh = 1;
                break;
            }
            umma::bar_expect_tx(&full[s], bytes);
            uint8_t *a = sa + s * C::SA_AL;
            uint8_t *b = sb + s * C::SB_AL;
            if (MODE == 0) {
                const int cblocks = g.cin / CBA;
                const int t = kb / cblocks, cb = kb % cblocks;
                int dy, dx;
                tap_offset(g.taps, t, dy, dx);
                umma::tma_load_4d(a, &tmA, cb * CBA, x0 + dx, y0 + dy, n, &full[s]);
                umma::tma_load_2d(b, &tmB, kb * CBA, co0, &full[s]);
            } else {
                const long long p0 = (long long)(kb0 + kb) * kKP;
                const int hw = g.H * g.W;
                const int pn = (int)(p0 / hw), pr = (int)(p0 % hw);
                const int py = pr / g.W, px = pr % g.W;
                int dy, dx;
                tap_offset(g.taps, tap, dy, dx);
                for (int j = 0; j < ga_valid; j++)
                    umma::tma_load_4d(a + j * kKP * C::RA, &tmA, co0 + j * CBA, px, py, pn, &full[s]);
                for (int j = 0; j < BN / CBB; j++)
                    umma::tma_load_4d(b + j * kKP * C::RB, &tmB, ci0 + j * CBB, px + dx, py + dy, pn, &full[s]);
            }
        }
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issue
        const uint32_t idesc = umma::make_idesc(128, BN, MODE, MODE);
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb % C::STAGES, round = kb / C::STAGES;
            if (!umma::bar_wait(&full[s], round & 1)) {
                fail_sh = 1;
                break;
            }
            umma::tc_fence_after();
            const uint32_t a0 = umma::smem_addr(sa + s * C::SA_AL);
            const uint32_t b0 = umma::smem_addr(sb + s * C::SB_AL);
#pragma unroll
            for (int kk = 0; kk < C::KSTEPS; kk++) {
                uint64_t ad, bd;
                if (MODE == 0) {
                    ad = umma::make_desc(a0 + kk * 32, 16, 8 * C::RA, C::RA);
                    bd = umma::make_desc(b0 + kk * 32, 16, 8 * C::RB, C::RB);
                } else {
                    ad = umma::make_desc(a0 + kk * 16 * C::RA, kKP * C::RA, 8 * C::RA, C::RA);
                    bd = umma::make_desc(b0 + kk * 16 * C::RB, kKP * C::RB, 8 * C::RB, C::RB);
                }
                umma::mma_bf16(tmem, ad, bd, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
            }
            umma::mma_commit(&empty[s]);
        }
        umma::mma_commit(&done);
    }
    __syncwarp();

    // ---- epilogue: accumulator rows are TMEM lanes (warp w: lanes 32w..)
    const bool got = umma::bar_wait(&done, 0);
    umma::tc_fence_after();
    const int row = warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    if (MODE == 0) {
        const int y = y0 + row / g.bw, x = x0 + row % g.bw;
        const size_t pix = ((size_t)n * g.H + y) * g.W + x;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            umma::tmem_ld16(trow + c0, v);
            const int co = co0 + c0;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                float t = v[i];
                if (g.bias)
                    t += g.bias[co + i];
                if (g.add)
                    t += __bfloat162float(g.add[pix * g.add_ld + co + i]);
                if (g.relu)
                    t = fmaxf(t, 0.f);
                if (g.mask && !(__bfloat162float(g.mask[pix * g.mask_ld + co + i]) > 0.f))
                    t = 0.f;
                v[i] = t;
            }
            if (g.out) {
                __align__(16) bf16 h[16];
#pragma unroll
                for (int i = 0; i < 16; i++)
                    h[i] = __float2bfloat16_rn(v[i]);
                uint4 *dst = reinterpret_cast<uint4 *>(g.out + pix * g.out_ld + g.out_coff + co);
                dst[0] = reinterpret_cast<const uint4 *>(h)[0];
                dst[1] = reinterpret_cast<const uint4 *>(h)[1];
            }
            if (g.out_f32) {
                float4 *dst = reinterpret_cast<float4 *>(g.out_f32 + pix * g.outf_ld + co);
#pragma unroll
                for (int i = 0; i < 4; i++)
                    dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            }
        }
    } else {
        const int co = co0 + row;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            umma::tmem_ld16(trow + c0, v);
            if (co < g.cout) {
                float *dst = g.dw + ((size_t)co * g.taps + tap) * g.cin + ci0 + c0;
#pragma unroll
                for (int i = 0; i < 16; i++)
                    atomicAdd(dst + i, v[i]);
            }
        }
    }
    if (threadIdx.x == 0 && (!got || fail_sh) && g.status)
        atomicExch(g.status, 1);
    umma::tc_fence_before();
    __syncthreads();
    if (warp == 0)
        umma::tmem_dealloc(tmem, C::TCOLS);
}

// Persistent forward / data-gradient GEMM (mode 0 geometry).  Each CTA
// walks tiles blockIdx.x, blockIdx.x + gridDim.x, ... of the 128-pixel x BN
// output; the K blocks of consecutive tiles flow through one TMA stage ring
// without a break, and the accumulator is double-buffered in tensor memory,
// so the epilogue of a tile overlaps the MMAs of the next.  Warps 0-3: the
// epilogue (warp w reads accumulator lanes 32w..32w+31); warp 4: tensor
// memory allocation and, in lane 0, the TMA producer; warp 5 lane 0: the MMA
// issuer.
constexpr int kPersistentThreads = 192;

template <int CB, int BN>
struct PersistCfg {
    static constexpr int R = CB * 2;
    static constexpr uint32_t SA = 128u * R, SB = (uint32_t)BN * R;
    static constexpr uint32_t STAGE = align1k(SA) + align1k(SB);
    static constexpr int ACC_COLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    static constexpr int TCOLS = 2 * ACC_COLS;  // two accumulators
    // one CTA per SM when its accumulators take all of tensor memory: then
    // the stage ring may use most of shared memory
    static constexpr uint32_t BUDGET = TCOLS == 512 ? 196608u : 98304u;
    static constexpr int STAGES = BUDGET / STAGE >= 6 ? 6 : (BUDGET / STAGE >= 2 ? (int)(BUDGET / STAGE) : 2);
    static constexpr uint32_t SMEM = STAGES * STAGE + 1024;
    static constexpr int KSTEPS = CB / 16;
};

template <int CB, int BN>
__global__ void __launch_bounds__(kPersistentThreads, 1)
    conv_gemm_persistent(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                         const GemmArgs g, int ntiles, int ntiles_n)
{
    using C = PersistCfg<CB, BN>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[C::STAGES], empty[C::STAGES], acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_sh;
    __shared__ int fail_store;
    volatile int &fail_sh = fail_store;  // set by any role that gave up waiting
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tx = g.W / g.bw, ty = g.H / g.bh;
    const int nk = g.taps * (g.cin / CB);
    const int cblocks = g.cin / CB;

    if (threadIdx.x == 0) {
        for (int i = 0; i < C::STAGES; i++) {
            umma::bar_init(&full[i], 1);
            umma::bar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            umma::bar_init(&acc_full[i], 1);
            umma::bar_init(&acc_empty[i], 4);  // one arrival per epilogue warp
        }
        umma::bar_fence_init();
        fail_sh = 0;
    }
    if (warp == 4) {
        umma::tmem_alloc(&tmem_sh, C::TCOLS);
        umma::tmem_relinquish();
    }
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
    const uint32_t tmem = tmem_sh;

    auto tile_coords = [&](int tile, int &n, int &y0, int &x0, int &co0) {
        const int tp = tile / ntiles_n, tn = tile % ntiles_n;
        n = tp / (tx * ty);
        const int r = tp % (tx * ty);
        y0 = (r / tx) * g.bh;
        x0 = (r % tx) * g.bw;
        co0 = tn * BN;
    };

    if (warp == 4) {
        if (lane == 0) {
            // ---- producer
            int gk = 0;
            for (int tile = blockIdx.x; tile < ntiles && !fail_sh; tile += gridDim.x) {
                int n, y0, x0, co0;
                tile_coords(tile, n, y0, x0, co0);
                for (int kb = 0; kb < nk; kb++, gk++) {
                    const int s = gk % C::STAGES, round = gk / C::STAGES;
                    if (round > 0 && !umma::bar_wait(&empty[s], (round - 1) & 1)) {
                        fail_sh = 1;
                        break;
                    }
                    umma::bar_expect_tx(&full[s], C::SA + C::SB);
                    uint8_t *a = smem + s * C::STAGE;
                    uint8_t *b = a + align1k(C::SA);
                    const int t = kb / cblocks, cb = kb % cblocks;
                    int dy, dx;
                    tap_offset(g.taps, t, dy, dx);
                    umma::tma_load_4d(a, &tmA, cb * CB, x0 + dx, y0 + dy, n, &full[s]);
                    umma::tma_load_2d(b, &tmB, kb * CB, co0, &full[s]);
                }
            }
        }
    } else if (warp == 5) {
        if (lane == 0) {
            // ---- MMA issue
            const uint32_t idesc = umma::make_idesc(128, BN, 0, 0);
            int gk = 0, it = 0;
            for (int tile = blockIdx.x; tile < ntiles && !fail_sh; tile += gridDim.x, it++) {
                const int ab = it & 1;
                if (it >= 2 && !umma::bar_wait(&acc_empty[ab], ((it >> 1) - 1) & 1)) {
                    fail_sh = 1;
                    break;
                }
                umma::tc_fence_after();
                const uint32_t acc = tmem + ab * C::ACC_COLS;
                for (int kb = 0; kb < nk; kb++, gk++) {
                    const int s = gk % C::STAGES, round = gk / C::STAGES;
                    if (!umma::bar_wait(&full[s], round & 1)) {
                        fail_sh = 1;
                        break;
                    }
                    umma::tc_fence_after();
                    const uint32_t a0 = umma::smem_addr(smem + s * C::STAGE);
                    const uint32_t b0 = a0 + align1k(C::SA);
#pragma unroll
                    for (int kk = 0; kk < C::KSTEPS; kk++) {
                        const uint64_t ad = umma::make_desc(a0 + kk * 32, 16, 8 * C::R, C::R);
                        const uint64_t bd = umma::make_desc(b0 + kk * 32, 16, 8 * C::R, C::R);
                        umma::mma_bf16(acc, ad, bd, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
                    }
                    umma::mma_commit(&empty[s]);
                }
                umma::mma_commit(&acc_full[ab]);
            }
        }
    } else {
        // ---- epilogue: warp w owns accumulator rows 32w..32w+31
        const int row = warp * 32 + lane;
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles && !fail_sh; tile += gridDim.x, it++) {
            const int ab = it & 1;
            if (!umma::bar_wait(&acc_full[ab], (it >> 1) & 1)) {
                fail_sh = 1;
                break;
            }
            umma::tc_fence_after();
            int n, y0, x0, co0;
            tile_coords(tile, n, y0, x0, co0);
            const int y = y0 + row / g.bw, x = x0 + row % g.bw;
            const size_t pix = ((size_t)n * g.H + y) * g.W + x;
            const uint32_t trow = tmem + ab * C::ACC_COLS + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                float v[16];
                umma::tmem_ld16(trow + c0, v);
                const int co = co0 + c0;
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    float t = v[i];
                    if (g.bias)
                        t += g.bias[co + i];
                    if (g.add)
                        t += __bfloat162float(g.add[pix * g.add_ld + co + i]);
                    if (g.relu)
                        t = fmaxf(t, 0.f);
                    if (g.mask && !(__bfloat162float(g.mask[pix * g.mask_ld + co + i]) > 0.f))
                        t = 0.f;
                    v[i] = t;
                }
                if (g.out) {
                    __align__(16) bf16 h[16];
#pragma unroll
                    for (int i = 0; i < 16; i++)
                        h[i] = __float2bfloat16_rn(v[i]);
                    uint4 *dst = reinterpret_cast<uint4 *>(g.out + pix * g.out_ld + g.out_coff + co);
                    dst[0] = reinterpret_cast<const uint4 *>(h)[0];
                    dst[1] = reinterpret_cast<const uint4 *>(h)[1];
                }
                if (g.out_f32) {
                    float4 *dst = reinterpret_cast<float4 *>(g.out_f32 + pix * g.outf_ld + co);
#pragma unroll
                    for (int i = 0; i < 4; i++)
                        dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                }
            }
            umma::tc_fence_before();
            __syncwarp();
            if (lane == 0)
                umma::bar_arrive(&acc_empty[ab]);
        }
    }
    __syncwarp();
    umma::tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && fail_sh && g.status)
        atomicExch(g.status, 1);
    if (warp == 4) {
        umma::tc_fence_after();
        umma::tmem_dealloc(tmem, C::TCOLS);
    }
}

// ------------------------------------------------------------------ host
namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encoder()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

CUtensorMapSwizzle swizzle_for(int cb) { return cb == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B; }

// NHWC activation tensor as a 4-D map {C, W, H, N}, box {cb, bw, bh, 1}.
bool map_nhwc(CUtensorMap *m, const void *base, int C, int W, int H, int N, int cb, int bw, int bh)
{
    cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {(cuuint32_t)cb, (cuuint32_t)bw, (cuuint32_t)bh, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return encoder()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(cb), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Row-major [rows][cols] bf16 matrix as a 2-D map, box {cb, brows}.
bool map_matrix(CUtensorMap *m, const void *base, int cols, int rows, int cb, int brows)
{
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)cb, (cuuint32_t)brows};
    cuuint32_t es[2] = {1, 1};
    return encoder()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(cb), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int MODE, int CBA, int CBB, int BN>
bool launch(const CUtensorMap &ta, const CUtensorMap &tb, const GemmArgs &g, dim3 grid, cudaStream_t s)
{
    using C = GemmCfg<MODE, CBA, CBB, BN>;
    auto k = conv_gemm_kernel<MODE, CBA, CBB, BN>;
    static bool configured = false;
    if (!configured) {
        if (!FMVD_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM)))
            return false;
        configured = true;
    }
    k<<<grid, 128, C::SMEM, s>>>(ta, tb, g);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

// pixel box of 'count' pixels on a W-wide image
void pixel_box(int W, int count, int &bw, int &bh)
{
    bw = W < count ? W : count;
    bh = count / bw;
}

template <int CB, int BN>
bool launch_persistent(const CUtensorMap &ta, const CUtensorMap &tb, const GemmArgs &g, int ntiles, int ntiles_n,
                       cudaStream_t s)
{
    using C = PersistCfg<CB, BN>;
    auto k = conv_gemm_persistent<CB, BN>;
    static int sms = 0;
    static bool configured = false;
    if (!configured) {
        int dev = 0;
        if (!FMVD_CHECK(cudaGetDevice(&dev)) ||
            !FMVD_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) ||
            !FMVD_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM)))
            return false;
        configured = true;
    }
    // CTAs per SM: tensor memory (512 columns) and shared memory allow
    const int by_tmem = 512 / C::TCOLS;
    const int by_smem = (int)(200u * 1024u / C::SMEM);
    const int per_sm = by_tmem < by_smem ? by_tmem : by_smem;
    int grid = sms * (per_sm < 1 ? 1 : per_sm);
    if (grid > ntiles)
        grid = ntiles;
    k<<<grid, kPersistentThreads, C::SMEM, s>>>(ta, tb, g, ntiles, ntiles_n);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

#define FMVD_BN_CASES(F) F(16) F(32) F(64) F(128) F(256)

template <int CB>
bool dispatch_persistent(int bn, const CUtensorMap &ta, const CUtensorMap &tb, const GemmArgs &g, int ntiles,
                         int ntiles_n, cudaStream_t s)
{
    switch (bn) {
#define X(B) \
    case B: return launch_persistent<CB, B>(ta, tb, g, ntiles, ntiles_n, s);
        FMVD_BN_CASES(X)
#undef X
    default: report_error("fmvd: unsupported GEMM N tile"); return false;
    }
}

template <int MODE, int CBA, int CBB>
bool dispatch_bn(int bn, const CUtensorMap &ta, const CUtensorMap &tb, const GemmArgs &g, dim3 grid, cudaStream_t s)
{
    switch (bn) {
#define X(B) \
    case B: return launch<MODE, CBA, CBB, B>(ta, tb, g, grid, s);
        FMVD_BN_CASES(X)
#undef X
    default: report_error("fmvd: unsupported GEMM N tile"); return false;
    }
}

} // namespace

bool conv_forward(const ConvDesc &c, cudaStream_t s)
{
    // D[pixel][co]: A = input activations (cin channels), B = weights [cout][taps][cin]
    if (!encoder()) {
        report_error("fmvd: cuTensorMapEncodeTiled is unavailable");
        return false;
    }
    const int cb = c.cin >= 64 ? 64 : 32;
    const int bn = c.cout > 256 ? 256 : c.cout;
    if (c.cin % cb || c.cout % bn || bn % 16 || (c.taps != 1 && c.taps != 9) || c.W % 8 || c.H * c.W < 128 ||
        (c.W < 128 ? 128 % c.W : c.W % 128) || (c.W < 128 && c.H % (128 / c.W))) {
        report_error("fmvd: unsupported convolution geometry");
        return false;
    }
    int bw, bh;
    pixel_box(c.W, 128, bw, bh);
    CUtensorMap ta, tb;
    if (!map_nhwc(&ta, c.in, c.cin, c.W, c.H, c.N, cb, bw, bh) ||
        !map_matrix(&tb, c.weight, c.taps * c.cin, c.cout, cb, bn)) {
        report_error("fmvd: tensor map encoding failed");
        return false;
    }
    GemmArgs g{};
    g.N = c.N;
    g.H = c.H;
    g.W = c.W;
    g.bw = bw;
    g.bh = bh;
    g.taps = c.taps;
    g.cin = c.cin;
    g.cout = c.cout;
    g.out = c.out;
    g.out_ld = c.out_ld ? c.out_ld : c.cout;
    g.out_coff = c.out_coff;
    g.out_f32 = c.out_f32;
    g.outf_ld = c.outf_ld ? c.outf_ld : c.cout;
    g.bias = c.bias;
    g.add = c.add;
    g.add_ld = c.add_ld ? c.add_ld : c.cout;
    g.mask = c.mask;
    g.mask_ld = c.mask_ld ? c.mask_ld : c.cout;
    g.relu = c.relu;
    g.status = c.status;
    const int ntiles_n = c.cout / bn;
    const int ntiles = c.N * (c.H / bh) * (c.W / bw) * ntiles_n;
    if (cb == 32 && bn <= 32) {
        // 32-channel operands with a narrow N: one CTA per tile keeps more
        // K blocks in flight per SM (measured faster on B200)
        const dim3 grid((unsigned)(ntiles / ntiles_n), (unsigned)ntiles_n, 1);
        return dispatch_bn<0, 32, 32>(bn, ta, tb, g, grid, s);
    }
    return cb == 64 ? dispatch_persistent<64>(bn, ta, tb, g, ntiles, ntiles_n, s)
                    : dispatch_persistent<32>(bn, ta, tb, g, ntiles, ntiles_n, s);
}

bool conv_wgrad(const WgradDesc &c, cudaStream_t s)
{
    // dW[co][t][ci] += sum_p G[p][co] X[p + off(t)][ci]
    if (!encoder()) {
        report_error("fmvd: cuTensorMapEncodeTiled is unavailable");
        return false;
    }
    const int cba = c.cout >= 64 ? 64 : 32;
    const int cbb = c.cin >= 64 ? 64 : 32;
    const int bn = c.cin > 256 ? 256 : c.cin;
    const long long pixels = (long long)c.N * c.H * c.W;
    if (c.cout % cba || c.cin % cbb || c.cin % bn || bn % 16 || (c.taps != 1 && c.taps != 9) ||
        (c.H * c.W) % kKP || (c.W < kKP ? kKP % c.W : c.W % kKP)) {
        report_error("fmvd: unsupported weight-gradient geometry");
        return false;
    }
    int bw, bh;
    pixel_box(c.W, kKP, bw, bh);
    CUtensorMap ta, tb;
    if (!map_nhwc(&ta, c.grad, c.cout, c.W, c.H, c.N, cba, bw, bh) ||
        !map_nhwc(&tb, c.in, c.cin, c.W, c.H, c.N, cbb, bw, bh)) {
        report_error("fmvd: tensor map encoding failed");
        return false;
    }
    const int total = (int)(pixels / kKP);
    const int co_tiles = (c.cout + 127) / 128;
    const int ci_tiles = c.cin / bn;
    // split K so that the grid covers the GPU a few times over
    const long long base = (long long)c.taps * co_tiles * ci_tiles;
    int kchunk = (int)((total * base + 1183) / 1184);
    if (kchunk < 16)
        kchunk = 16;
    if (kchunk > total)
        kchunk = total;
    GemmArgs g{};
    g.N = c.N;
    g.H = c.H;
    g.W = c.W;
    g.bw = bw;
    g.bh = bh;
    g.taps = c.taps;
    g.cin = c.cin;
    g.cout = c.cout;
    g.kchunk = kchunk;
    g.dw = c.dw;
    g.status = c.status;
    const dim3 grid((unsigned)(c.taps * co_tiles), (unsigned)((total + kchunk - 1) / kchunk), (unsigned)ci_tiles);
    if (cba == 64)
        return cbb == 64 ? dispatch_bn<1, 64, 64>(bn, ta, tb, g, grid, s) : dispatch_bn<1, 64, 32>(bn, ta, tb, g, grid, s);
    return cbb == 64 ? dispatch_bn<1, 32, 64>(bn, ta, tb, g, grid, s) : dispatch_bn<1, 32, 32>(bn, ta, tb, g, grid, s);
}

} // namespace unet
} // namespace fmvd
