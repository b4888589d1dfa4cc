// Complex arithmetic and register-resident power-of-two DFTs (2, 4, 8, 16)
// for sm_100a; the warp FFT (warp_fft.cuh) builds its lines from them.
//
// Direction: DIR = -1 computes X[m] = sum_n x[n] exp(-2 pi i m n / N),
// DIR = +1 the unnormalised inverse.  Twiddle tables hold exp(-2 pi i n / N)
// computed on the host in double precision.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fmvd {

// ---------------------------------------------------------------- complex
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * (c + DIR i s)
template <int DIR>
__device__ __forceinline__ float2 cmul_cs(float2 a, float c, float s)
{
    return DIR < 0 ? make_float2(a.x * c + a.y * s, a.y * c - a.x * s)
                   : make_float2(a.x * c - a.y * s, a.y * c + a.x * s);
}
// a * (DIR i)
template <int DIR>
__device__ __forceinline__ float2 crot(float2 a)
{
    return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
// twiddle from the forward table, conjugated for the inverse direction
template <int DIR>
__device__ __forceinline__ float2 ctw(float2 a, float2 t)
{
    return DIR < 0 ? cmul(a, t) : make_float2(a.x * t.x + a.y * t.y, a.y * t.x - a.x * t.y);
}

// --------------------------------------------------------- small DFTs
// cos / sin of multiples of pi / 8 (mathematical constants)
constexpr float kC8 = 0.70710678118654752440f;   // cos(pi/4)
constexpr float kC16 = 0.92387953251128675613f;  // cos(pi/8)
constexpr float kS16 = 0.38268343236508977173f;  // sin(pi/8)

template <int DIR>
__device__ __forceinline__ void dft2(float2 &a0, float2 &a1)
{
    float2 t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}

template <int DIR>
__device__ __forceinline__ void dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3)
{
    float2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
    float2 t2 = cadd(a1, a3), t3 = crot<DIR>(csub(a1, a3));
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, t3);
    a3 = csub(t1, t3);
}

template <int R, int DIR>
struct Dft;

template <int DIR>
struct Dft<2, DIR> {
    static __device__ __forceinline__ void run(float2 *v) { dft2<DIR>(v[0], v[1]); }
};

template <int DIR>
struct Dft<4, DIR> {
    static __device__ __forceinline__ void run(float2 *v) { dft4<DIR>(v[0], v[1], v[2], v[3]); }
};

// 8 = 4 (stride 2) x 2
template <int DIR>
struct Dft<8, DIR> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        dft4<DIR>(v[0], v[2], v[4], v[6]);
        dft4<DIR>(v[1], v[3], v[5], v[7]);
        // odd half times w8^m, m = 0..3
        v[3] = cmul_cs<DIR>(v[3], kC8, kC8);
        v[5] = crot<DIR>(v[5]);
        v[7] = cmul_cs<DIR>(v[7], -kC8, kC8);
        float2 o[8];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            o[m] = cadd(v[2 * m], v[2 * m + 1]);
            o[m + 4] = csub(v[2 * m], v[2 * m + 1]);
        }
#pragma unroll
        for (int m = 0; m < 8; m++)
            v[m] = o[m];
    }
};

// 16 = 4 (stride 4) x 4
template <int DIR>
struct Dft<16, DIR> {
    static __device__ __forceinline__ void run(float2 *v)
    {
#pragma unroll
        for (int b = 0; b < 4; b++)
            dft4<DIR>(v[b], v[4 + b], v[8 + b], v[12 + b]);
        // Y_b[m1] lives in v[4 * m1 + b]; multiply by w16^(b m1)
        v[5] = cmul_cs<DIR>(v[5], kC16, kS16);      // b=1 m1=1: w^1
        v[9] = cmul_cs<DIR>(v[9], kC8, kC8);        // b=1 m1=2: w^2
        v[13] = cmul_cs<DIR>(v[13], kS16, kC16);    // b=1 m1=3: w^3
        v[6] = cmul_cs<DIR>(v[6], kC8, kC8);        // b=2 m1=1: w^2
        v[10] = crot<DIR>(v[10]);                   // b=2 m1=2: w^4
        v[14] = cmul_cs<DIR>(v[14], -kC8, kC8);     // b=2 m1=3: w^6
        v[7] = cmul_cs<DIR>(v[7], kS16, kC16);      // b=3 m1=1: w^3
        v[11] = cmul_cs<DIR>(v[11], -kC8, kC8);     // b=3 m1=2: w^6
        v[15] = cmul_cs<DIR>(v[15], -kC16, -kS16);  // b=3 m1=3: w^9
        float2 o[16];
#pragma unroll
        for (int m1 = 0; m1 < 4; m1++) {
            float2 a0 = v[4 * m1], a1 = v[4 * m1 + 1], a2 = v[4 * m1 + 2], a3 = v[4 * m1 + 3];
            dft4<DIR>(a0, a1, a2, a3);
            o[m1] = a0;
            o[m1 + 4] = a1;
            o[m1 + 8] = a2;
            o[m1 + 12] = a3;
        }
#pragma unroll
        for (int m = 0; m < 16; m++)
            v[m] = o[m];
    }
};

} // namespace fmvd
