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

// ------------------------------------------- forward DFTs of length 3..8
// SmallDft<R>::run(z): z[k] = sum_n z[n] exp(-2 pi i n k / R), in place, with
// R-specific short forms for 3, 4, 5 and 8 and a direct form for 6 and 7.
// cos / sin (2 pi j / R) (mathematical constants)
constexpr float kC3 = -0.5f, kS3 = 0.86602540378443864676f;
constexpr float kC5a = 0.30901699437494742410f, kC5b = -0.80901699437494742410f;
constexpr float kS5a = 0.95105651629515357212f, kS5b = 0.58778525229247312917f;
// cos / sin (2 pi j / R) for R = 6, 7 (a switch that folds away once j is a
// compile-time constant after unrolling)
template <int R>
__device__ __forceinline__ void unit_root(int j, float &c, float &s)
{
    if constexpr (R == 6) {
        constexpr float h = 0.86602540378443864676f;
        switch (j) {
        case 0: c = 1.f; s = 0.f; break;
        case 1: c = 0.5f; s = h; break;
        case 2: c = -0.5f; s = h; break;
        case 3: c = -1.f; s = 0.f; break;
        case 4: c = -0.5f; s = -h; break;
        default: c = 0.5f; s = -h; break;
        }
    } else {
        static_assert(R == 7, "direct forms for 6 and 7 only");
        constexpr float c1 = 0.62348980185873353053f, c2 = -0.22252093395631440429f, c3 = -0.90096886790241912624f;
        constexpr float s1 = 0.78183148246802980871f, s2 = 0.97492791218182360702f, s3 = 0.43388373911755812048f;
        switch (j) {
        case 0: c = 1.f; s = 0.f; break;
        case 1: c = c1; s = s1; break;
        case 2: c = c2; s = s2; break;
        case 3: c = c3; s = s3; break;
        case 4: c = c3; s = -s3; break;
        case 5: c = c2; s = -s2; break;
        default: c = c1; s = -s1; break;
        }
    }
}

// -i * b
__device__ __forceinline__ float2 cmul_negi(float2 b) { return make_float2(b.y, -b.x); }

template <int R>
struct SmallDft;

template <>
struct SmallDft<3> {
    static __device__ __forceinline__ void run(float2 *z)
    {
        const float2 t1 = cadd(z[1], z[2]);
        const float2 d = csub(z[1], z[2]);
        const float2 t2 = make_float2(z[0].x + kC3 * t1.x, z[0].y + kC3 * t1.y);
        const float2 u = cmul_negi(make_float2(kS3 * d.x, kS3 * d.y));
        z[0] = cadd(z[0], t1);
        z[1] = cadd(t2, u);
        z[2] = csub(t2, u);
    }
};

template <>
struct SmallDft<4> {
    static __device__ __forceinline__ void run(float2 *z) { dft4<-1>(z[0], z[1], z[2], z[3]); }
};

template <>
struct SmallDft<5> {
    static __device__ __forceinline__ void run(float2 *z)
    {
        const float2 t1 = cadd(z[1], z[4]), t2 = cadd(z[2], z[3]);
        const float2 t3 = csub(z[1], z[4]), t4 = csub(z[2], z[3]);
        const float2 a1 = make_float2(z[0].x + kC5a * t1.x + kC5b * t2.x, z[0].y + kC5a * t1.y + kC5b * t2.y);
        const float2 a2 = make_float2(z[0].x + kC5b * t1.x + kC5a * t2.x, z[0].y + kC5b * t1.y + kC5a * t2.y);
        const float2 b1 = make_float2(kS5a * t3.x + kS5b * t4.x, kS5a * t3.y + kS5b * t4.y);
        const float2 b2 = make_float2(kS5b * t3.x - kS5a * t4.x, kS5b * t3.y - kS5a * t4.y);
        z[0] = cadd(z[0], cadd(t1, t2));
        const float2 m1 = cmul_negi(b1), m2 = cmul_negi(b2);
        z[1] = cadd(a1, m1);
        z[4] = csub(a1, m1);
        z[2] = cadd(a2, m2);
        z[3] = csub(a2, m2);
    }
};

template <int R>
struct DirectDft {
    static __device__ __forceinline__ void run(float2 *z)
    {
        float2 o[R];
#pragma unroll
        for (int k = 0; k < R; k++) {
            float2 acc = z[0];
#pragma unroll
            for (int n = 1; n < R; n++) {
                float c, s;
                unit_root<R>((n * k) % R, c, s);
                // z[n] * (cos - i sin)
                acc.x += z[n].x * c + z[n].y * s;
                acc.y += z[n].y * c - z[n].x * s;
            }
            o[k] = acc;
        }
#pragma unroll
        for (int k = 0; k < R; k++)
            z[k] = o[k];
    }
};

template <>
struct SmallDft<6> : DirectDft<6> {};
template <>
struct SmallDft<7> : DirectDft<7> {};
template <>
struct SmallDft<8> {
    static __device__ __forceinline__ void run(float2 *z) { Dft<8, -1>::run(z); }
};

} // namespace fmvd
