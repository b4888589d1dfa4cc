// Shared-memory batched 1-D complex FFT for sm_100a.
//
// A thread block holds F independent length-N transforms in shared memory
// (split real / imaginary float arrays, padded against bank conflicts) and runs
// a Stockham autosort schedule N = R_0 * R_1 * ... * R_L: each stage is a
// register-resident radix-R butterfly (R in {2, 3, 4, 5, 8, 16} or a generic
// odd prime up to 31), with the data exchanged through shared memory between
// stages.  The first stage may take its input from registers and the last
// stage may leave its output in registers; both use the same "edge" pattern
//     v[b * R + r] = x[f][j + r * N / R],  q = tid + b * NT, f = q / (N/R), j = q % (N/R)
// so the output of one transform feeds the next without a shared-memory trip
// when both use the same edge radix, and element-wise work (kernel multiply,
// data/blur ratio, estimate update) runs on registers in between.
//
// Direction: DIR = -1 computes X[m] = sum_n x[n] exp(-2 pi i m n / N),
// DIR = +1 the unnormalised inverse.  Twiddles come from a table of
// exp(-2 pi i n / N) computed on the host in double precision.
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
// cos / sin of multiples of pi / 8 and of 2 pi / 3, 2 pi / 5 (mathematical constants)
constexpr float kC8 = 0.70710678118654752440f;   // cos(pi/4)
constexpr float kC16 = 0.92387953251128675613f;  // cos(pi/8)
constexpr float kS16 = 0.38268343236508977173f;  // sin(pi/8)
constexpr float kS3 = 0.86602540378443864676f;   // sin(2 pi/3)
constexpr float kC51 = 0.30901699437494742410f;  // cos(2 pi/5)
constexpr float kC52 = -0.80901699437494742410f; // cos(4 pi/5)
constexpr float kS51 = 0.95105651629515357212f;  // sin(2 pi/5)
constexpr float kS52 = 0.58778525229247312917f;  // sin(4 pi/5)

// cos / sin (2 pi k / R) for the generic odd radices.  Each translation unit
// that includes this header gets its own copy; the host fills it through
// upload_odd_radix_table() once per device before the first launch.
struct OddRadixTable {
    float c[32][32];
    float s[32][32];
};
static __constant__ OddRadixTable g_odd;

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

template <int DIR>
struct Dft<3, DIR> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        float2 t = cadd(v[1], v[2]);
        float2 u = crot<DIR>(csub(v[1], v[2]));
        u = make_float2(u.x * kS3, u.y * kS3);
        float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
        v[0] = cadd(v[0], t);
        v[1] = cadd(m, u);
        v[2] = csub(m, u);
    }
};

template <int DIR>
struct Dft<5, DIR> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        float2 b1 = make_float2(v[0].x + kC51 * t1.x + kC52 * t2.x, v[0].y + kC51 * t1.y + kC52 * t2.y);
        float2 b2 = make_float2(v[0].x + kC52 * t1.x + kC51 * t2.x, v[0].y + kC52 * t1.y + kC51 * t2.y);
        float2 d1 = crot<DIR>(make_float2(kS51 * t3.x + kS52 * t4.x, kS51 * t3.y + kS52 * t4.y));
        float2 d2 = crot<DIR>(make_float2(kS52 * t3.x - kS51 * t4.x, kS52 * t3.y - kS51 * t4.y));
        v[0] = cadd(v[0], cadd(t1, t2));
        v[1] = cadd(b1, d1);
        v[4] = csub(b1, d1);
        v[2] = cadd(b2, d2);
        v[3] = csub(b2, d2);
    }
};

// generic odd prime radix: direct evaluation with symmetric pairs
template <int R, int DIR>
struct Dft {
    static_assert(R % 2 == 1 && R <= 31, "unsupported radix");
    static __device__ __forceinline__ void run(float2 *v)
    {
        constexpr int H = (R - 1) / 2;
        float2 sp[H], sm[H];
#pragma unroll
        for (int k = 1; k <= H; k++) {
            sp[k - 1] = cadd(v[k], v[R - k]);
            sm[k - 1] = csub(v[k], v[R - k]);
        }
        float2 o[R];
        float2 x0 = v[0];
        o[0] = x0;
#pragma unroll
        for (int k = 0; k < H; k++)
            o[0] = cadd(o[0], sp[k]);
#pragma unroll
        for (int m = 1; m <= H; m++) {
            float2 re = x0, im = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 1; k <= H; k++) {
                const int km = (k * m) % R;
                const float c = g_odd.c[R][km], s = g_odd.s[R][km];
                re.x += c * sp[k - 1].x;
                re.y += c * sp[k - 1].y;
                im.x += s * sm[k - 1].x;
                im.y += s * sm[k - 1].y;
            }
            float2 d = crot<DIR>(im);
            o[m] = cadd(re, d);
            o[R - m] = csub(re, d);
        }
#pragma unroll
        for (int m = 0; m < R; m++)
            v[m] = o[m];
    }
};

// ------------------------------------------------------------ schedules
// Radix schedule for length N: edge radix E at both ends, middle factors in
// between (powers of two first as 4/8/16, then odd primes ascending).
struct Schedule {
    int n;
    int count;
    int r[16];
};

__host__ __device__ constexpr int largest_pow2_edge(int n)
{
    return (n % 256 == 0) ? 16 : (n % 64 == 0) ? 8 : (n % 16 == 0) ? 4 : (n % 4 == 0) ? 2 : 1;
}

__host__ __device__ constexpr Schedule make_schedule(int n)
{
    Schedule s{n, 0, {0}};
    int e = largest_pow2_edge(n);
    int m = n;
    if (e > 1) {
        s.r[s.count++] = e;
        m /= e * e;
    }
    int mid[16] = {0};
    int nm = 0;
    while (m % 16 == 0) { mid[nm++] = 16; m /= 16; }
    while (m % 8 == 0) { mid[nm++] = 8; m /= 8; }
    while (m % 4 == 0) { mid[nm++] = 4; m /= 4; }
    while (m % 2 == 0) { mid[nm++] = 2; m /= 2; }
    for (int f = 3; m > 1 && f <= 31; f += 2)
        while (m % f == 0) { mid[nm++] = f; m /= f; }
    for (int i = 0; i < nm; i++)
        s.r[s.count++] = mid[i];
    if (e > 1)
        s.r[s.count++] = e;
    if (m != 1)
        s.count = -1;  // prime factor above 31: unsupported
    return s;
}

template <int N>
struct Sched {
    static constexpr Schedule s = make_schedule(N);
    static constexpr int count = s.count;
    static constexpr int edge = s.r[0];
    static_assert(count > 1, "unsupported FFT length");
    template <int I>
    __host__ __device__ static constexpr int radix() { return s.r[I]; }
    template <int I>
    __host__ __device__ static constexpr int ns()
    {
        int p = 1;
        for (int i = 0; i < I; i++)
            p *= s.r[i];
        return p;
    }
};

// ------------------------------------------------------------- smem map
// Row-of-transform stride and element position inside the padded buffer.
template <int N>
struct SmemLayout {
    static constexpr int ld = N + (N >> 4) + 1;
    static __device__ __forceinline__ int at(int f, int n) { return f * ld + n + (n >> 4); }
    __host__ __device__ static constexpr int floats(int F) { return F * ld; }
};

// -------------------------------------------------------------- stages
// One Stockham stage.  Input from shared memory, or from registers (edge
// pattern) when IN_REGS; output to shared memory, or to registers (edge
// pattern) when OUT_REGS.  Edge stages need NT to divide their butterfly
// count; middle stages run ceil(butterflies / NT) rounds with a bound check.
template <int N, int F, int NT, int R, int NS, int DIR, bool IN_REGS, bool OUT_REGS>
__device__ __forceinline__ void fft_stage(float *sre, float *sim, float2 *v, const float2 *__restrict__ tw)
{
    using L = SmemLayout<N>;
    constexpr int NB = F * N / R;       // butterflies in this stage
    constexpr bool EXACT = (NB % NT == 0);
    static_assert(EXACT || (!IN_REGS && !OUT_REGS), "edge stages need NT | butterflies");
    constexpr int Q = (NB + NT - 1) / NT;
    const int tid = threadIdx.x;
    float2 w[Q * R];
    float2 *x = (IN_REGS || OUT_REGS) ? v : w;
    if (!IN_REGS) {
#pragma unroll
        for (int b = 0; b < Q; b++) {
            const int q = tid + b * NT;
            if (EXACT || q < NB) {
                const int f = q / (N / R), j = q % (N / R);
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const int a = L::at(f, j + r * (N / R));
                    x[b * R + r] = make_float2(sre[a], sim[a]);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int b = 0; b < Q; b++) {
        const int q = tid + b * NT;
        if (EXACT || q < NB) {
            const int j = q % (N / R);
            if (NS > 1) {
                const int k = j % NS;
#pragma unroll
                for (int r = 1; r < R; r++)
                    x[b * R + r] = ctw<DIR>(x[b * R + r], __ldg(tw + r * k * (N / (NS * R))));
            }
            Dft<R, DIR>::run(x + b * R);
        }
    }
    if (!OUT_REGS) {
#pragma unroll
        for (int b = 0; b < Q; b++) {
            const int q = tid + b * NT;
            if (EXACT || q < NB) {
                const int f = q / (N / R), j = q % (N / R);
                const int base = (j / NS) * NS * R + (j % NS);
#pragma unroll
                for (int m = 0; m < R; m++) {
                    const int a = L::at(f, base + m * NS);
                    sre[a] = x[b * R + m].x;
                    sim[a] = x[b * R + m].y;
                }
            }
        }
        __syncthreads();
    }
}

// Runs stages [I, count) of the schedule; the first (I == 0) may take its
// input from registers, the last always leaves its output in registers.
template <int N, int F, int NT, int DIR, int I, bool FIRST_IN_REGS>
struct StageRunner {
    static __device__ __forceinline__ void run(float *sre, float *sim, float2 *v, const float2 *tw)
    {
        using S = Sched<N>;
        constexpr int R = S::template radix<I>();
        constexpr int NS = S::template ns<I>();
        constexpr bool LAST = (I == S::count - 1);
        fft_stage<N, F, NT, R, NS, DIR, (I == 0) && FIRST_IN_REGS, LAST>(sre, sim, v, tw);
        if constexpr (!LAST)
            StageRunner<N, F, NT, DIR, I + 1, FIRST_IN_REGS>::run(sre, sim, v, tw);
    }
};

// Full transform.  On entry the data is in shared memory (natural order) or,
// with FIRST_IN_REGS, in registers in the edge pattern.  On exit the result
// is in registers in the edge pattern and shared memory is free to reuse
// (all threads have passed a barrier after their last shared-memory read).
template <int N, int F, int NT, int DIR, bool FIRST_IN_REGS>
__device__ __forceinline__ void fft(float *sre, float *sim, float2 *v, const float2 *__restrict__ tw)
{
    StageRunner<N, F, NT, DIR, 0, FIRST_IN_REGS>::run(sre, sim, v, tw);
}

// Number of complex values per thread for the edge pattern.
template <int N, int F, int NT>
struct Edge {
    static constexpr int R = Sched<N>::edge;
    static constexpr int E = F * N / NT;
    static constexpr int Q = E / R;
    // transform index and element index of register slot e = b * R + m
    static __device__ __forceinline__ void pos(int e, int &f, int &n)
    {
        const int b = e / R, m = e % R;
        const int q = threadIdx.x + b * NT;
        f = q / (N / R);
        n = q % (N / R) + m * (N / R);
    }
};

// Registers (edge pattern) -> shared memory (natural order).  The caller
// synchronises before reading the shared memory.
template <int N, int F, int NT>
__device__ __forceinline__ void regs_to_smem(float *sre, float *sim, const float2 *v)
{
    using L = SmemLayout<N>;
    using EG = Edge<N, F, NT>;
#pragma unroll
    for (int e = 0; e < EG::E; e++) {
        int f, n;
        EG::pos(e, f, n);
        const int a = L::at(f, n);
        sre[a] = v[e].x;
        sim[a] = v[e].y;
    }
}

} // namespace fmvd
