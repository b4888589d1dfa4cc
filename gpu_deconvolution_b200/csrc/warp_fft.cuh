// Warp-level complex FFT of length N <= 1024 for sm_100a.
//
// A group of T lanes (T <= 32, inside one warp) owns one length-N line,
// N = T * E with T <= E, lane t holding v[m] = x[t + T m] (m < E) in registers.
// The transform is the four-step factorisation N = T x E:
//   1. an E-point DFT in registers over m              -> Y[t][k1]
//   2. twiddle Y[t][k1] *= w_N^(t k1)                  (table, coalesced)
//   3. transpose through shared memory: lane t takes the sequences
//      k1 = t + T s (s < E/T); positions are XOR-swizzled so that both the
//      write and the read of the transpose are free of bank conflicts
//   4. a T-point DFT in registers over t for each of those sequences
// giving X[k1 + E k2], which lands in lane t as v[m] = X[t + T m] again: the
// same pattern as the input, so element-wise work between a transform and the
// next runs on registers, and lines load and store with coalesced accesses.
// The only synchronisation is __syncwarp (the group lives in one warp).
#pragma once

#include "fft_engine.cuh"
#include "rl_kernels.h"

namespace fmvd {

// cos / sin (pi m / 16), m = 0..8 (mathematical constants)
constexpr float kC32[9] = {1.0f,
                           0.98078528040323044913f,
                           0.92387953251128675613f,
                           0.83146961230254523708f,
                           0.70710678118654752440f,
                           0.55557023301960222474f,
                           0.38268343236508977173f,
                           0.19509032201612826785f,
                           0.0f};

// a * w32^m for compile-time m (w32 = exp(DIR 2 pi i / 32))
template <int DIR, int M>
__device__ __forceinline__ float2 mul_w32(float2 a)
{
    constexpr int m = M % 32;
    if constexpr (m == 0) {
        return a;
    } else if constexpr (m == 8) {
        return crot<DIR>(a);
    } else if constexpr (m == 16) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (m == 24) {
        return crot<-DIR>(a);
    } else {
        // angle = 2 pi m / 32 = pi m / 16; reduce to the first quadrant
        constexpr int q = m / 8, r = m % 8;
        // cos, sin of pi r / 16
        constexpr float c = kC32[r], s = kC32[8 - r];
        // rotate by the quadrant first, then by r
        float2 b = a;
        if constexpr (q == 1)
            b = crot<DIR>(a);
        else if constexpr (q == 2)
            b = make_float2(-a.x, -a.y);
        else if constexpr (q == 3)
            b = crot<-DIR>(a);
        return cmul_cs<DIR>(b, c, s);
    }
}

// 32 = 8 (stride 4) x 4
template <int DIR>
struct Dft<32, DIR> {
    template <int N2>
    static __device__ __forceinline__ void twiddle_column(float2 *v)
    {
        // A[n2][k1] at v[4 k1 + n2] times w32^(n2 k1)
        v[4 * 1 + N2] = mul_w32<DIR, N2 * 1>(v[4 * 1 + N2]);
        v[4 * 2 + N2] = mul_w32<DIR, N2 * 2>(v[4 * 2 + N2]);
        v[4 * 3 + N2] = mul_w32<DIR, N2 * 3>(v[4 * 3 + N2]);
        v[4 * 4 + N2] = mul_w32<DIR, N2 * 4>(v[4 * 4 + N2]);
        v[4 * 5 + N2] = mul_w32<DIR, N2 * 5>(v[4 * 5 + N2]);
        v[4 * 6 + N2] = mul_w32<DIR, N2 * 6>(v[4 * 6 + N2]);
        v[4 * 7 + N2] = mul_w32<DIR, N2 * 7>(v[4 * 7 + N2]);
    }
    static __device__ __forceinline__ void run(float2 *v)
    {
        // step A: four 8-point DFTs over n1 of x[4 n1 + n2]
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) {
            float2 t[8];
#pragma unroll
            for (int n1 = 0; n1 < 8; n1++)
                t[n1] = v[4 * n1 + n2];
            Dft<8, DIR>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < 8; k1++)
                v[4 * k1 + n2] = t[k1];
        }
        // step B: twiddles w32^(n2 k1)
        twiddle_column<1>(v);
        twiddle_column<2>(v);
        twiddle_column<3>(v);
        // step C: eight 4-point DFTs over n2 -> X[k1 + 8 k2]
        float2 o[32];
#pragma unroll
        for (int k1 = 0; k1 < 8; k1++) {
            float2 a0 = v[4 * k1], a1 = v[4 * k1 + 1], a2 = v[4 * k1 + 2], a3 = v[4 * k1 + 3];
            dft4<DIR>(a0, a1, a2, a3);
            o[k1] = a0;
            o[k1 + 8] = a1;
            o[k1 + 16] = a2;
            o[k1 + 24] = a3;
        }
#pragma unroll
        for (int m = 0; m < 32; m++)
            v[m] = o[m];
    }
};

// Lanes per line for each length: the largest power of two T with T * T <= N.
__host__ __device__ constexpr int warp_fft_lanes(int n)
{
    return n >= 1024 ? 32 : n >= 256 ? 16 : n >= 64 ? 8 : 4;
}

template <int N>
struct WarpFft {
    static_assert(N >= 16 && N <= 1024 && (N & (N - 1)) == 0, "warp FFT lengths are powers of two 16..1024");
    static constexpr int T = warp_fft_lanes(N);
    static constexpr int E = N / T;
    static constexpr int S = E / T;
    // Shared-memory floats per group (real and imaginary planes).  The group
    // size T is added so that the G = 32 / T groups of a warp start T banks
    // apart: with the XOR swizzle below, every transpose write and read of a
    // whole warp then touches 32 distinct banks.
    static constexpr int group_floats = 2 * N + T;

    // Position of transpose element (k1, t) inside a group's buffer.
    static __device__ __forceinline__ int tpos(int k1, int t) { return k1 * T + (t ^ (k1 & (T - 1))); }

    // Twiddle table layout (per length N, built on the host, float2):
    //   [j * T + t]       = w_N^(R8 j t)   for j < J   (R8 = min(E, kWarpTwiddleRun), J = E / R8)
    //   [J * T + t]       = w_N^t
    // Lane t forms w_N^(t k1), k1 = R8 j + b, as table[j] * (w_N^t)^b with the
    // powers b < R8 by repeated multiplication: J + 1 loads per transform
    // instead of E - 1, and at most R8 rounding steps per twiddle.
    static constexpr int R8 = E < kWarpTwiddleRun ? E : kWarpTwiddleRun;
    static constexpr int J = E / R8;
    static constexpr int table_size = (J + 1) * T;

    // In-place transform of v (lane pattern v[m] = x[t + T m]).
    // tw: twiddle table above.  The transpose buffer element p lives at
    // bre[p * STRIDE] / bim[p * STRIDE] (this group's shared memory); t: lane
    // index inside the group.
    // Transpose buffer element p at bre[p * STRIDE] / bim[p * STRIDE].
    template <int STRIDE>
    struct StridedAddr {
        __device__ __forceinline__ int operator()(int p) const { return p * STRIDE; }
    };

    template <int DIR, int STRIDE = 1>
    static __device__ __forceinline__ void run(float2 *v, const float2 *__restrict__ tw, float *bre, float *bim,
                                               int t)
    {
        run_addr<DIR>(v, tw, bre, bim, t, StridedAddr<STRIDE>());
    }

    // Step 2: v[k1] *= w_N^(t k1), k1 < E (table entries times a recurrence).
    template <int DIR>
    static __device__ __forceinline__ void twiddle(float2 *v, const float2 *__restrict__ tw, int t)
    {
        const float2 w1 = __ldg(tw + J * T + t);
        float2 wp[R8];
        wp[0] = make_float2(1.f, 0.f);
        if (R8 > 1)
            wp[1] = w1;
#pragma unroll
        for (int b = 2; b < R8; b++)
            wp[b] = cmul(wp[b - 1], w1);
#pragma unroll
        for (int j = 0; j < J; j++) {
            const float2 wj = j == 0 ? make_float2(1.f, 0.f) : __ldg(tw + j * T + t);
#pragma unroll
            for (int b = 0; b < R8; b++) {
                const int k1 = j * R8 + b;
                if (k1 == 0)
                    continue;
                const float2 w = j == 0 ? wp[b] : (b == 0 ? wj : cmul(wj, wp[b]));
                v[k1] = ctw<DIR>(v[k1], w);
            }
        }
    }

    // Step 4 output order: X[t + T s + E k2] is in v[s * T + k2]; move it to v[s + S k2].
    static __device__ __forceinline__ void reorder(float2 *v)
    {
        if constexpr (S > 1) {
            float2 o[E];
#pragma unroll
            for (int s = 0; s < S; s++)
#pragma unroll
                for (int k2 = 0; k2 < T; k2++)
                    o[s + S * k2] = v[s * T + k2];
#pragma unroll
            for (int m = 0; m < E; m++)
                v[m] = o[m];
        }
    }

    // Complex (float2) elements of a group's padded transpose buffer: row k1
    // of T + 1 entries, so that the writes (lane t, fixed k1) and the reads
    // (lane t, row t + T s) are both free of bank conflicts with 64-bit
    // accesses at compile-time offsets.
    static constexpr int padded_f2 = E * (T + 1);
    static constexpr int padded_floats = ((2 * padded_f2 + 3) / 4) * 4;  // 16-byte multiple

    struct Nothing {
        __device__ __forceinline__ void operator()() const {}
    };

    // The transform with the transpose through the padded float2 buffer buf.
    // after_read() runs once every lane has read its transpose elements back,
    // when buf is free for other use until the next transform.
    template <int DIR, typename AfterRead = Nothing>
    static __device__ __forceinline__ void run_padded(float2 *v, const float2 *__restrict__ tw, float2 *buf, int t,
                                                      const AfterRead &after_read = AfterRead())
    {
        Dft<E, DIR>::run(v);
        twiddle<DIR>(v, tw, t);
        float2 *wr = buf + t;
#pragma unroll
        for (int k1 = 0; k1 < E; k1++)
            wr[k1 * (T + 1)] = v[k1];
        __syncwarp();
        const float2 *rd = buf + t * (T + 1);
#pragma unroll
        for (int s = 0; s < S; s++)
#pragma unroll
            for (int j = 0; j < T; j++)
                v[s * T + j] = rd[s * T * (T + 1) + j];
        __syncwarp();
        after_read();
#pragma unroll
        for (int s = 0; s < S; s++)
            Dft<T, DIR>::run(v + s * T);
        reorder(v);
    }

    // Same, with the transpose element p at buf[addr(p)] (float2).
    template <int DIR, typename Addr>
    static __device__ __forceinline__ void run_addr2(float2 *v, const float2 *__restrict__ tw, float2 *buf, int t,
                                                     const Addr &addr)
    {
        Dft<E, DIR>::run(v);
        twiddle<DIR>(v, tw, t);
#pragma unroll
        for (int k1 = 0; k1 < E; k1++)
            buf[addr(tpos(k1, t))] = v[k1];
        __syncwarp();
#pragma unroll
        for (int s = 0; s < S; s++) {
            const int k1 = t + T * s;
#pragma unroll
            for (int j = 0; j < T; j++)
                v[s * T + j] = buf[addr(tpos(k1, j))];
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < S; s++)
            Dft<T, DIR>::run(v + s * T);
        reorder(v);
    }

    // Same, with the transpose buffer element p at bre[addr(p)] / bim[addr(p)].
    template <int DIR, typename Addr>
    static __device__ __forceinline__ void run_addr(float2 *v, const float2 *__restrict__ tw, float *bre, float *bim,
                                                    int t, const Addr &addr)
    {
        Dft<E, DIR>::run(v);
        twiddle<DIR>(v, tw, t);
#pragma unroll
        for (int k1 = 0; k1 < E; k1++) {
            const int p = addr(tpos(k1, t));
            bre[p] = v[k1].x;
            bim[p] = v[k1].y;
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < S; s++) {
            const int k1 = t + T * s;
#pragma unroll
            for (int j = 0; j < T; j++) {
                const int p = addr(tpos(k1, j));
                v[s * T + j] = make_float2(bre[p], bim[p]);
            }
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < S; s++)
            Dft<T, DIR>::run(v + s * T);
        reorder(v);
    }
};

} // namespace fmvd
