// Affine trilinear resampler and transformed weight mask on sm_100a.
//
// Replaces transform_cuda_8/16 of the reference (fmvd_transform.impl.cu:77-224),
// which binds the source to a 3-D texture and fetches every target voxel with
// hardware trilinear filtering.  Here the source lives in plain device memory
// (rows padded to 16 bytes) described by a 3-D TMA tensor map.  Each CTA
// resamples a 32 x 8 tile of a stack of up to 16 consecutive target planes:
// since the map is affine, every stack's source footprint has the same shape,
// so the host sizes one box that covers it (with slack for rounding), one
// thread issues a single cp.async.bulk.tensor load of that brick into shared
// memory (out-of-volume texels arrive as zeros, the texture's border colour),
// and the threads interpolate every plane of the stack from shared memory.
// Consecutive target planes sample overlapping source footprints, so one
// brick per stack moves a fraction of the bytes of one brick per plane.  The
// interpolation follows the texture unit's linear filter: texel centres at
// i + 0.5, weights held with 8 fractional bits, values normalised by
// 2^bits - 1; output quantised as the reference does,
// (sample)(v * 2^bits + 0.5) through a 32-bit integer.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <mutex>
#include <thread>
#include <vector>

#include "fmvd_internal.h"
#include "transform_kernels.h"

namespace fmvd {

namespace {

constexpr int TX = 32, TY = 8;  // target tile
#ifndef FMVD_RESAMPLE_STACK
#define FMVD_RESAMPLE_STACK 16
#endif
constexpr int kMaxStack = FMVD_RESAMPLE_STACK;  // target planes per CTA, at most

struct Mat {
    float m[12];
};

// rx = m0 x + m1 y + m2 z + m3 (fmvd_transform.impl.cu:41-43), same evaluation
// order; z may be passed as the float it converts to (a whole number)
template <typename Z>
__device__ __forceinline__ void apply(const Mat &M, int x, int y, Z z, float &rx, float &ry, float &rz)
{
    rx = M.m[0] * x + M.m[1] * y + M.m[2] * z + M.m[3];
    ry = M.m[4] * x + M.m[5] * y + M.m[6] * z + M.m[7];
    rz = M.m[8] * x + M.m[9] * y + M.m[10] * z + M.m[11];
}

// Texel index and 1/256-quantised weight along one axis for source position r
// (the reference fetches at r + 0.5 in unnormalised texture coordinates; the
// filter works at xB = coordinate - 0.5).  The fractional part is rounded to
// the nearest 1/256, halves up: q = floor((xB) * 256 + 0.5) in 1/256 texels,
// texel q >> 8 (a floor, also below zero), weight (q mod 256) / 256.
__device__ __forceinline__ void tex_axis(float r, int &i, float &a)
{
    // the reference forms r + 0.5 in double and converts to float: the exact
    // sum rounded once to float, which is what one float addition gives
    const float u = __fadd_rn(r, 0.5f);
    const float xb = __fsub_rn(u, 0.5f);
    // xb * 256 is exact, so the fused form rounds the same sum as
    // (xb * 256) + 0.5 would; one conversion (to int, rounding down) instead
    // of two floors and a conversion
    const int q = __float2int_rd(__fmaf_rn(xb, 256.0f, 0.5f));
    i = q >> 8;
    // (q & 255) / 256 exactly: those bits placed as the lowest mantissa bits
    // of 2^15 (whose unit in the last place is 1/256), then 2^15 taken away
    a = __int_as_float(0x47000000 | (q & 255)) - 32768.0f;
}

// A sample as a float: the integer value is placed in the low mantissa bits
// of 2^23 and 2^23 taken away (exact for values below 2^23), so the
// conversion uses the FP32 pipe instead of the conversion unit.
template <typename S>
__device__ __forceinline__ float sample_value(S v)
{
    return __int_as_float(0x4B000000 | (uint32_t)v) - 8388608.0f;
}

// Trilinear blend of the corner samples t[c] (c = x + 2 y + 4 z offsets)
// with the upper-corner weights ax, ay, az, in sample units; the texture's
// normalised value is this times 1 / (2^bits - 1).
__device__ __forceinline__ float blend(const float *t, float ax, float ay, float az)
{
    const float bx0 = 1.f - ax, by0 = 1.f - ay, bz0 = 1.f - az;
    return bz0 * (by0 * (bx0 * t[0] + ax * t[1]) + ay * (bx0 * t[2] + ax * t[3])) +
           az * (by0 * (bx0 * t[4] + ax * t[5]) + ay * (bx0 * t[6] + ax * t[7]));
}

template <typename S, int BITS>
__device__ __forceinline__ S quantise(float v)
{
    // (SAMPLE)(v * 2^BITS + 0.5) as the reference compiles it: float product,
    // double sum, conversion through a 32-bit unsigned integer, so a fetch of
    // exactly 1.0 wraps to 0 (measured on the B200).  The product is exact
    // (a power of two) and below 2^23, where adding 0.5 in float is exact
    // too, so float arithmetic gives the same integer.
    const float q = __fadd_rn(v * (float)(1 << BITS), 0.5f);
    return (S)__float2uint_rz(q);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Output of a resampler launch: target samples, the float blend, or both.
constexpr int kOutSamples = 1, kOutFloat = 2;

template <typename S, int BITS, int OUT>
__global__ void __launch_bounds__(TX *TY) resample_tma(const __grid_constant__ CUtensorMap tmap,
                                                       const S *__restrict__ src, int w, int h, int d, size_t pitch,
                                                       int tw, int th, int z0, int nz, int kz, const Mat M, int bx,
                                                       int by, int bz, S *__restrict__ out, float *__restrict__ outf,
                                                       int *__restrict__ status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int origin[3];
    // 0: no brick (every texel from global memory); 1: brick, each load
    // checked against it; 2: brick holding every texel of the tile stack
    __shared__ int mode;
    const S *brick = reinterpret_cast<const S *>(smem_raw);
    constexpr int XALIGN = 16 / sizeof(S);
    // this CTA: a TX x TY tile of the kz target planes zb .. zb + kz - 1
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, zb = z0 + blockIdx.z * kz;
    const int zn = min(kz, z0 + nz - zb);
    const int tid = threadIdx.x;

    if (tid < 32) {
        // lane c (mod 8): corner c of the tile stack.  Each source coordinate
        // is monotonic in x, y and z separately (an affine map evaluated with
        // monotonic roundings), and so are the texel indices, so the corners
        // bound every index of the stack.
        const int c = tid & 7;
        float r[3];
        apply(M, x0 + (c & 1) * (TX - 1), y0 + ((c >> 1) & 1) * (TY - 1), (float)(zb + (c >> 2) * (zn - 1)), r[0],
              r[1], r[2]);
        float mn[3] = {r[0], r[1], r[2]};
#pragma unroll
        for (int o = 1; o < 8; o <<= 1)
#pragma unroll
            for (int k = 0; k < 3; k++)
                mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
        // brick origin: one texel below the footprint, x rounded down to the
        // 16-byte boundary a TMA copy needs
        int ox = (int)floorf(mn[0]) - 1;
        ox = (ox >= 0) ? (ox / XALIGN) * XALIGN : -(((-ox) + XALIGN - 1) / XALIGN) * XALIGN;
        const int oy = (int)floorf(mn[1]) - 1;
        const int oz = (int)floorf(mn[2]) - 1;
        // the corners' texels inside the brick with one texel to spare on
        // each side (room for a different rounding of the same coordinate)
        int ix, iy, iz;
        float a;
        tex_axis(r[0], ix, a);
        tex_axis(r[1], iy, a);
        tex_axis(r[2], iz, a);
        const bool inside = ix - ox >= 1 && ix - ox + 2 < bx && iy - oy >= 1 && iy - oy + 2 < by && iz - oz >= 1 &&
                            iz - oz + 2 < bz;
        const bool all_inside = __all_sync(0xffffffffu, inside);
        if (tid == 0) {
            origin[0] = ox;
            origin[1] = oy;
            origin[2] = oz;
            const uint32_t bar_a = smem_u32(&bar);
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            const uint32_t bytes = (uint32_t)(bx * by * bz * sizeof(S));
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes) : "memory");
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
                    smem_u32(smem_raw)),
                "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(ox), "r"(oy), "r"(oz), "r"(bar_a)
                : "memory");
            // bounded wait for the brick (phase 0), by this thread alone: the
            // others wait at the block barrier below, where they take no issue
            // slots, and the barrier orders the brick's arrival before their
            // reads
            uint32_t done = 0;
            for (int spin = 0; spin < (1 << 22) && !done; spin++) {
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(done)
                    : "r"(bar_a)
                    : "memory");
                if (!done && spin > 64)
                    __nanosleep(64);
            }
            mode = done ? (all_inside ? 2 : 1) : 0;
            if (!done)
                atomicExch(status, 1);
        }
    }
    __syncthreads();  // the origin and mode are written and the brick has landed (or the wait gave up)
    const int ox = origin[0], oy = origin[1], oz = origin[2];
    const int md = mode;

    const int x = x0 + (tid % TX), y = y0 + (tid / TX);
    if (x >= tw || y >= th)
        return;
    const float inv = 1.0f / (float)((1 << BITS) - 1);
    const size_t plane = (size_t)th * tw;
    const size_t first = ((size_t)(zb - z0) * th + y) * tw + x;
    S *o = (OUT & kOutSamples) ? out + first : nullptr;
    float *of = (OUT & kOutFloat) ? outf + first : nullptr;
    const auto emit = [&](float raw) {
        if constexpr ((OUT & kOutSamples) != 0) {
            *o = quantise<S, BITS>(raw * inv);
            o += plane;
        }
        if constexpr ((OUT & kOutFloat) != 0) {
            *of = raw;
            of += plane;
        }
    };
    float zf = (float)zb;  // the target plane as a float: whole numbers, exact
    if (md == 2) {
        // every texel of the stack is in the brick: no per-voxel checks
        const int sy = bx, sz = bx * by;
#pragma unroll 2
        for (int k = 0; k < zn; k++, zf += 1.0f) {
            float rx, ry, rz;
            apply(M, x, y, zf, rx, ry, rz);
            int ix, iy, iz;
            float ax, ay, az;
            tex_axis(rx, ix, ax);
            tex_axis(ry, iy, ay);
            tex_axis(rz, iz, az);
            const S *b0 = brick + ((iz - oz) * by + (iy - oy)) * bx + (ix - ox);
            float t[8];
#pragma unroll
            for (int c = 0; c < 8; c++)
                t[c] = sample_value(b0[(c >> 2) * sz + ((c >> 1) & 1) * sy + (c & 1)]);
            emit(blend(t, ax, ay, az));
        }
        return;
    }
#pragma unroll 1
    for (int k = 0; k < zn; k++, zf += 1.0f) {
        float rx, ry, rz;
        apply(M, x, y, zf, rx, ry, rz);
        int ix, iy, iz;
        float ax, ay, az;
        tex_axis(rx, ix, ax);
        tex_axis(ry, iy, ay);
        tex_axis(rz, iz, az);
        const int lx = ix - ox, ly = iy - oy, lz = iz - oz;
        float t[8];
        if (md == 1 && (unsigned)lx < (unsigned)(bx - 1) && (unsigned)ly < (unsigned)(by - 1) &&
            (unsigned)lz < (unsigned)(bz - 1)) {
            const S *b0 = brick + (lz * by + ly) * bx + lx;
#pragma unroll
            for (int c = 0; c < 8; c++)
                t[c] = sample_value(b0[((c >> 2) * by + ((c >> 1) & 1)) * bx + (c & 1)]);
        } else {
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const int sx = ix + (c & 1), sy = iy + ((c >> 1) & 1), sz = iz + (c >> 2);
                const bool in = sx >= 0 && sx < w && sy >= 0 && sy < h && sz >= 0 && sz < d;
                t[c] = in ? sample_value(__ldg(src + ((size_t)sz * h + sy) * pitch + sx)) : 0.f;
            }
        }
        emit(blend(t, ax, ay, az));
    }
}

// fmvd_transform.cu:19-67
__global__ void mask_kernel(float *__restrict__ out, int z, int w, int h, int d, float zspacing, int tw, int th,
                            float border, const Mat M)
{
    const int x = threadIdx.x + blockIdx.x * blockDim.x;
    const int y = threadIdx.y + blockIdx.y * blockDim.y;
    if (x >= tw || y >= th)
        return;
    float rx, ry, rz;
    apply(M, x, y, z, rx, ry, rz);
    float v = 0.f;
    if (!(rx < 0 || rx >= w || ry < 0 || ry >= h || rz < 0 || rz >= d)) {
        const float pi = 3.14159265358979323846f;
        float dx = rx < w / 2 ? rx : w - rx;
        float dy = ry < h / 2 ? ry : h - ry;
        float dz = rz < d / 2 ? rz : d - rz;
        dz *= zspacing;
        v = 1.f;
        if (dx < border)
            v *= 0.5f * (1 - cosf(dx / border * pi));
        if (dy < border)
            v *= 0.5f * (1 - cosf(dy / border * pi));
        if (dz < border)
            v *= 0.5f * (1 - cosf(dz / border * pi));
    }
    out[(size_t)y * tw + x] = v;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
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

int ceil_i(float v) { return (int)ceilf(v); }

} // namespace

// Source volume in device memory: d planes of h rows, row pitch 'pitch'
// samples (a multiple of 16 bytes).
bool resample_device(int bits, const void *d_src, size_t pitch, int w, int h, int d, int tw, int th, int z0, int nz,
                     const float *h_inverse, void *d_out, float *d_outf, int *d_status, cudaStream_t s)
{
    const size_t es = bits == 16 ? 2 : 1;
    Mat M;
    memcpy(M.m, h_inverse, sizeof(M.m));
    const int xalign = (int)(16 / es);
    // box covering the footprint of a stack of kz tiles: extent + 2 texels
    // for the filter and slack, one more so that every texel of the stack is
    // in the brick with one to spare, plus the alignment of the x origin; kz
    // is the deepest stack (16, 8, 4, 2 or 1 target planes) whose box fits
    int box[3] = {0, 0, 0};
    int kz = kMaxStack;
    size_t smem = 0;
    bool boxes_ok = false;
    for (; kz >= 1; kz /= 2) {
        for (int a = 0; a < 3; a++) {
            const float ext = fabsf(M.m[4 * a]) * (TX - 1) + fabsf(M.m[4 * a + 1]) * (TY - 1) +
                              fabsf(M.m[4 * a + 2]) * (kz - 1);
            box[a] = ceil_i(ext) + 5;
        }
        box[0] = ((box[0] + xalign - 1 + xalign - 1) / xalign) * xalign;
        // shared-memory banks: a brick row is 16 bytes times an odd number
        // and a plane an odd number of rows, so lanes that step through rows
        // or planes (rotated views) spread over 8 banks instead of 2 or 4
        if ((box[0] / xalign) % 2 == 0)
            box[0] += xalign;
        box[1] |= 1;
        smem = (size_t)box[0] * box[1] * box[2] * es;
        boxes_ok = box[0] <= 256 && box[1] <= 256 && box[2] <= 256 && smem <= 96 * 1024;
        if (boxes_ok)
            break;
    }
    if (kz < 1)
        kz = 1;

    CUtensorMap tmap;
    memset(&tmap, 0, sizeof(tmap));
    bool use_tma = boxes_ok && encode_fn() != nullptr;
    if (use_tma) {
        cuuint64_t gdim[3] = {(cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)d};
        cuuint64_t gstride[2] = {(cuuint64_t)(pitch * es), (cuuint64_t)(pitch * es * h)};
        cuuint32_t bdim[3] = {(cuuint32_t)box[0], (cuuint32_t)box[1], (cuuint32_t)box[2]};
        cuuint32_t estride[3] = {1, 1, 1};
        CUresult r = encode_fn()(&tmap, bits == 16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8, 3,
                                 const_cast<void *>(d_src), gdim, gstride, bdim, estride,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        use_tma = (r == CUDA_SUCCESS);
    }
    dim3 grid((tw + TX - 1) / TX, (th + TY - 1) / TY, (nz + kz - 1) / kz);
    if (!use_tma) {  // no brick fits (extreme scaling): every voxel takes the direct path
        resample_direct(bits, d_src, pitch, w, h, d, tw, th, z0, nz, h_inverse, d_out, d_outf, s);
        return FMVD_CHECK(cudaGetLastError());
    }
    const int mode = (d_out ? kOutSamples : 0) | (d_outf ? kOutFloat : 0);
    if (mode == 0)
        return true;
    const auto launch = [&](auto kern, auto *src_typed, auto *out_typed) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, TX * TY, smem, s>>>(tmap, src_typed, w, h, d, pitch, tw, th, z0, nz, kz, M, box[0], box[1],
                                         box[2], out_typed, d_outf, d_status);
        rl_count_launch(1);
    };
    if (bits == 16) {
        using S = unsigned short;
        const S *sp = (const S *)d_src;
        S *op = (S *)d_out;
        if (mode == kOutSamples)
            launch(resample_tma<S, 16, kOutSamples>, sp, op);
        else if (mode == kOutFloat)
            launch(resample_tma<S, 16, kOutFloat>, sp, op);
        else
            launch(resample_tma<S, 16, kOutSamples | kOutFloat>, sp, op);
    } else {
        using S = unsigned char;
        const S *sp = (const S *)d_src;
        S *op = (S *)d_out;
        if (mode == kOutSamples)
            launch(resample_tma<S, 8, kOutSamples>, sp, op);
        else if (mode == kOutFloat)
            launch(resample_tma<S, 8, kOutFloat>, sp, op);
        else
            launch(resample_tma<S, 8, kOutSamples | kOutFloat>, sp, op);
    }
    return FMVD_CHECK(cudaGetLastError());
}

bool mask_device(float *d_out, int z, int w, int h, int d, float zspacing, int tw, int th, float border,
                 const float *h_inverse, cudaStream_t s)
{
    Mat M;
    memcpy(M.m, h_inverse, sizeof(M.m));
    dim3 threads(32, 8);
    dim3 grid((tw + 31) / 32, (th + 7) / 8);
    mask_kernel<<<grid, threads, 0, s>>>(d_out, z, w, h, d, zspacing, tw, th, border, M);
    rl_count_launch(1);
    return FMVD_CHECK(cudaGetLastError());
}

// Direct-gather variant (no TMA brick): every texel read from global memory.
template <typename S, int BITS>
__global__ void resample_direct_kernel(const S *__restrict__ src, int w, int h, int d, size_t pitch, int tw, int th,
                                       int z0, const Mat M, S *__restrict__ out, float *__restrict__ outf)
{
    const int x = blockIdx.x * TX + (threadIdx.x % TX), y = blockIdx.y * TY + (threadIdx.x / TX);
    const int z = z0 + blockIdx.z;
    if (x >= tw || y >= th)
        return;
    float rx, ry, rz;
    apply(M, x, y, z, rx, ry, rz);
    int ix, iy, iz;
    float ax, ay, az;
    tex_axis(rx, ix, ax);
    tex_axis(ry, iy, ay);
    tex_axis(rz, iz, az);
    const float inv = 1.0f / (float)((1 << BITS) - 1);
    float t[8];
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const int sx = ix + (c & 1), sy = iy + ((c >> 1) & 1), sz = iz + (c >> 2);
        const bool in = sx >= 0 && sx < w && sy >= 0 && sy < h && sz >= 0 && sz < d;
        t[c] = in ? sample_value(__ldg(src + ((size_t)sz * h + sy) * pitch + sx)) : 0.f;
    }
    const float raw = blend(t, ax, ay, az);
    const size_t oi = ((size_t)blockIdx.z * th + y) * tw + x;
    if (out)
        out[oi] = quantise<S, BITS>(raw * inv);
    if (outf)
        outf[oi] = raw;
}

void resample_direct(int bits, const void *d_src, size_t pitch, int w, int h, int d, int tw, int th, int z0, int nz,
                     const float *h_inverse, void *d_out, float *d_outf, cudaStream_t s)
{
    Mat M;
    memcpy(M.m, h_inverse, sizeof(M.m));
    dim3 grid((tw + TX - 1) / TX, (th + TY - 1) / TY, nz);
    if (bits == 16)
        resample_direct_kernel<unsigned short, 16><<<grid, TX * TY, 0, s>>>(
            (const unsigned short *)d_src, w, h, d, pitch, tw, th, z0, M, (unsigned short *)d_out, d_outf);
    else
        resample_direct_kernel<unsigned char, 8><<<grid, TX * TY, 0, s>>>(
            (const unsigned char *)d_src, w, h, d, pitch, tw, th, z0, M, (unsigned char *)d_out, d_outf);
    rl_count_launch(1);
}

size_t source_pitch(int bits, int w)
{
    const size_t a = bits == 16 ? 8 : 16;
    return ((size_t)w + a - 1) / a * a;
}

// Host copies of many bytes split over a few threads (a single thread moves
// only a few GB/s from pageable memory).
void host_copy(void *dst, const void *src, size_t bytes)
{
    constexpr size_t kPiece = size_t(4) << 20;
    const int nt = (int)std::min<size_t>(8, bytes / kPiece);
    if (nt < 2) {
        memcpy(dst, src, bytes);
        return;
    }
    const size_t part = (bytes + nt - 1) / nt;
    std::vector<std::thread> th;
    for (int i = 1; i < nt; i++) {
        const size_t o = part * i, n = std::min(part, bytes - o);
        th.emplace_back([=] { memcpy((char *)dst + o, (const char *)src + o, n); });
    }
    memcpy(dst, src, std::min(part, bytes));
    for (auto &t : th)
        t.join();
}

// Upload of d source planes (host pointers, any host memory) into the
// pitched device volume: planes are packed into two pinned staging buffers in
// turn, each staging buffer's copy to the device running while the host
// packs the next.
// Pinned staging buffers of the host-memory entry points, kept for the life
// of the process: pinning host memory costs far more than the copies through
// it, so the buffers are allocated once and grown when a call needs more.
// Callers hold the lock for the whole call (the reference's host-memory
// entry points are not reentrant either).
namespace {
std::mutex g_stage_lock;
void *g_stage[4] = {nullptr, nullptr, nullptr, nullptr};
size_t g_stage_bytes[4] = {0, 0, 0, 0};
} // namespace

std::unique_lock<std::mutex> staging_lock() { return std::unique_lock<std::mutex>(g_stage_lock); }

void *staging_buffer(int i, size_t bytes)
{
    if (g_stage[i] && !pinned_still_valid(g_stage[i])) {  // released by a device reset
        g_stage[i] = nullptr;
        g_stage_bytes[i] = 0;
    }
    if (g_stage_bytes[i] < bytes) {
        cudaFreeHost(g_stage[i]);
        g_stage[i] = nullptr;
        g_stage_bytes[i] = 0;
        if (!FMVD_CHECK(cudaMallocHost(&g_stage[i], bytes)))
            return nullptr;
        g_stage_bytes[i] = bytes;
    }
    return g_stage[i];
}

bool upload_planes(const void *const *h_planes, int w, int h, int d, size_t es, size_t pitch, void *d_src,
                   cudaStream_t s)
{
    const size_t row = (size_t)w * es, plane = row * h;
    int per = (int)(((size_t)16 << 20) / (plane ? plane : 1));
    per = per < 1 ? 1 : (per > d ? (d > 0 ? d : 1) : per);
    void *stage[2] = {staging_buffer(0, plane * per), staging_buffer(1, plane * per)};
    cudaEvent_t done[2] = {nullptr, nullptr};
    bool ok = stage[0] && stage[1];
    for (int k = 0; k < 2 && ok; k++)
        ok = FMVD_CHECK(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming));
    bool used[2] = {false, false};
    for (int z0 = 0, k = 0; ok && z0 < d; z0 += per, k ^= 1) {
        const int n = d - z0 < per ? d - z0 : per;
        if (used[k])
            ok = FMVD_CHECK(cudaEventSynchronize(done[k]));  // the staging buffer's last copy has landed
        if (ok) {
            // planes over a few threads
            const int nt = std::max(1, std::min(8, (int)((plane * n) >> 22)));
            std::vector<std::thread> th;
            auto part = [&, k, z0, n, nt](int id) {
                for (int i = id; i < n; i += nt)
                    memcpy((char *)stage[k] + plane * i, h_planes[z0 + i], plane);
            };
            for (int id = 1; id < nt; id++)
                th.emplace_back(part, id);
            part(0);
            for (auto &t : th)
                t.join();
        }
        ok = ok && FMVD_CHECK(cudaMemcpy2DAsync((char *)d_src + pitch * h * z0 * es, pitch * es, stage[k], row, row,
                                                (size_t)h * n, cudaMemcpyHostToDevice, s)) &&
             FMVD_CHECK(cudaEventRecord(done[k], s));
        used[k] = true;
    }
    if (ok)
        ok = FMVD_CHECK(cudaStreamSynchronize(s));
    else
        cudaStreamSynchronize(s);
    for (int k = 0; k < 2; k++)
        if (done[k])
            cudaEventDestroy(done[k]);
    return ok;
}

// transform_cuda_* (fmvd_transform.impl.cu:77-224): upload, optional mask of
// plane td/2, resample in chunks of planes with download and file write of
// one chunk overlapping the resampling of the next.  Every device buffer,
// event and stream is released on every path (the pinned staging buffers are
// the process-wide ones above).
void transform_file(int bits, const void *const *h_planes, int w, int h, int d, int tw, int th, int td,
                    const float *h_inverse, const char *outfile, int masks, int border, float zspacing,
                    const char *maskfile)
{
    auto lock = staging_lock();
    const size_t es = bits == 16 ? 2 : 1;
    const size_t pitch = source_pitch(bits, w);
    void *d_src = nullptr;
    int *d_status = nullptr;
    cudaStream_t s = nullptr;
    bool ok = FMVD_CHECK(cudaMalloc(&d_src, pitch * h * d * es)) && FMVD_CHECK(cudaMalloc(&d_status, sizeof(int))) &&
              FMVD_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) &&
              FMVD_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), s)) &&
              upload_planes(h_planes, w, h, d, es, pitch, d_src, s);

    if (ok && masks) {
        float *d_m = nullptr;
        std::vector<float> hm((size_t)tw * th);
        if (FMVD_CHECK(cudaMalloc(&d_m, sizeof(float) * tw * th)) &&
            mask_device(d_m, td / 2, w, h, d, zspacing, tw, th, (float)border, h_inverse, s) &&
            FMVD_CHECK(cudaMemcpyAsync(hm.data(), d_m, sizeof(float) * tw * th, cudaMemcpyDeviceToHost, s)) &&
            FMVD_CHECK(cudaStreamSynchronize(s))) {
            FILE *f = fopen(maskfile, "wb");
            if (f) {
                fwrite(hm.data(), sizeof(float), (size_t)tw * th, f);
                fclose(f);
            } else {
                report_error("fmvd: could not open the mask file");
            }
        }
        cudaFree(d_m);
    }

    FILE *out = ok ? fopen(outfile, "wb") : nullptr;
    if (ok && !out)
        report_error("fmvd: could not open the output file");
    if (out) {
        const size_t plane_bytes = (size_t)tw * th * es;
        // The reference writes an unfilled slot ahead of the data when td < 2.
        if (td < 2) {
            std::vector<char> zero(plane_bytes, 0);
            for (int i = 0; i < 2 - td; i++)
                fwrite(zero.data(), 1, plane_bytes, out);
        }
        int chunk = (int)(((size_t)16 << 20) / (plane_bytes ? plane_bytes : 1));
        if (chunk < 1)
            chunk = 1;
        if (chunk > td)
            chunk = td > 0 ? td : 1;
        void *d_out[2] = {nullptr, nullptr};
        void *h_out[2] = {staging_buffer(2, plane_bytes * chunk), staging_buffer(3, plane_bytes * chunk)};
        cudaEvent_t ev[2] = {nullptr, nullptr};
        ok = ok && h_out[0] && h_out[1];
        for (int k = 0; k < 2 && ok; k++)
            ok = FMVD_CHECK(cudaMalloc(&d_out[k], plane_bytes * chunk)) &&
                 FMVD_CHECK(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
        int pending_k = -1, pending_n = 0;
        for (int z0 = 0, k = 0; ok && z0 < td; z0 += chunk, k ^= 1) {
            const int n = td - z0 < chunk ? td - z0 : chunk;
            ok = resample_device(bits, d_src, pitch, w, h, d, tw, th, z0, n, h_inverse, d_out[k], nullptr, d_status,
                                 s) &&
                 FMVD_CHECK(cudaMemcpyAsync(h_out[k], d_out[k], plane_bytes * n, cudaMemcpyDeviceToHost, s)) &&
                 FMVD_CHECK(cudaEventRecord(ev[k], s));
            if (ok && pending_k >= 0) {
                ok = FMVD_CHECK(cudaEventSynchronize(ev[pending_k]));
                fwrite(h_out[pending_k], 1, plane_bytes * pending_n, out);
            }
            pending_k = k;
            pending_n = n;
        }
        if (ok && pending_k >= 0) {
            ok = FMVD_CHECK(cudaEventSynchronize(ev[pending_k]));
            fwrite(h_out[pending_k], 1, plane_bytes * pending_n, out);
        }
        fclose(out);
        cudaStreamSynchronize(s);
        for (int k = 0; k < 2; k++) {
            cudaFree(d_out[k]);
            if (ev[k])
                cudaEventDestroy(ev[k]);
        }
    }
    if (d_status) {
        int status = 0;
        if (s)
            cudaStreamSynchronize(s);
        if (cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && status)
            report_error("fmvd: a resampler brick load did not complete in time");
    }
    if (s)
        cudaStreamDestroy(s);
    cudaFree(d_src);
    cudaFree(d_status);
}

} // namespace fmvd
