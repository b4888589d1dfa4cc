/* C/OpenMP port of the reference per-plane Richardson-Lucy update
 * (TEST INFRASTRUCTURE: the CPU baseline that bench.py times, and a second,
 * float32 checker for the tests).  Nothing in the product links it.
 *
 * It follows the reference loop (fmvd_deconvolve.impl.cpp:247-284) with the
 * element-wise semantics of fmvd_deconvolve_cuda.cu:13-414 and
 * fmvd_deconvolve_cuda.impl.cu:14-197:
 *   estimate = 10 * nViews on the padded fftH x fftW plane
 *   per iteration, per view v in order:
 *     b = conv(e, K_v) ; t = b > 1 ? d_v / b : b ; r = conv(t, Khat_v)
 *     e = e + w_v * (e * r - e)
 *   crop, clip at 2^bits - 1, truncate.
 * The circular convolutions use a project-written mixed-radix FFT (radix 2,
 * 3, 4, 5 and generic odd) in float32: two real planes share one complex
 * transform (real part = plane z, imaginary part = plane z + 1), which is
 * exact for real kernels.  OpenMP distributes plane pairs over threads.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

typedef struct { float re, im; } cpx;

/* ------------------------------------------------------------------ FFT */
typedef struct {
    int n;
    int nstages;
    int radix[32];
    cpx *tw;        /* exp(-2 pi i k / n), k < n */
} fft_plan;

static int fft_plan_init(fft_plan *p, int n)
{
    p->n = n;
    p->nstages = 0;
    int m = n;
    while (m % 4 == 0) { p->radix[p->nstages++] = 4; m /= 4; }
    while (m % 2 == 0) { p->radix[p->nstages++] = 2; m /= 2; }
    for (int f = 3; m > 1; f += 2)
        while (m % f == 0) { p->radix[p->nstages++] = f; m /= f; }
    p->tw = (cpx *)malloc(sizeof(cpx) * n);
    for (int k = 0; k < n; k++) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        p->tw[k].re = (float)cos(a);
        p->tw[k].im = (float)sin(a);
    }
    return 0;
}

static void fft_plan_free(fft_plan *p) { free(p->tw); }

/* Stockham autosort pass: x (n) -> y (n); sign = -1 forward, +1 inverse.
 * Ns = product of the radices already applied. */
static void fft_pass(const fft_plan *p, const cpx *x, cpx *y, int R, int Ns, int sign)
{
    int n = p->n;
    int nb = n / R;
    cpx v[32];
    for (int j = 0; j < nb; j++) {
        int k = j % Ns;
        for (int r = 0; r < R; r++) {
            cpx a = x[j + r * nb];
            /* twiddle exp(sign * 2 pi i r k / (Ns R)) */
            int idx = (int)(((long)r * k * (n / (Ns * R))) % n);
            cpx t = p->tw[idx];
            if (sign > 0) t.im = -t.im;
            v[r].re = a.re * t.re - a.im * t.im;
            v[r].im = a.re * t.im + a.im * t.re;
        }
        cpx o[32];
        if (R == 2) {
            o[0].re = v[0].re + v[1].re; o[0].im = v[0].im + v[1].im;
            o[1].re = v[0].re - v[1].re; o[1].im = v[0].im - v[1].im;
        } else if (R == 4) {
            cpx a0 = { v[0].re + v[2].re, v[0].im + v[2].im };
            cpx a1 = { v[0].re - v[2].re, v[0].im - v[2].im };
            cpx a2 = { v[1].re + v[3].re, v[1].im + v[3].im };
            cpx a3 = { v[1].re - v[3].re, v[1].im - v[3].im };
            /* multiply a3 by sign * i */
            cpx a3r = { -sign * a3.im, sign * a3.re };
            o[0].re = a0.re + a2.re; o[0].im = a0.im + a2.im;
            o[2].re = a0.re - a2.re; o[2].im = a0.im - a2.im;
            o[1].re = a1.re + a3r.re; o[1].im = a1.im + a3r.im;
            o[3].re = a1.re - a3r.re; o[3].im = a1.im - a3r.im;
        } else {
            /* direct odd-radix DFT */
            for (int m = 0; m < R; m++) {
                float sr = 0.f, si = 0.f;
                for (int r = 0; r < R; r++) {
                    int idx = (int)(((long)r * m % R) * (n / R));
                    cpx t = p->tw[idx];
                    if (sign > 0) t.im = -t.im;
                    sr += v[r].re * t.re - v[r].im * t.im;
                    si += v[r].re * t.im + v[r].im * t.re;
                }
                o[m].re = sr; o[m].im = si;
            }
        }
        int base = (j / Ns) * Ns * R + k;
        for (int r = 0; r < R; r++)
            y[base + r * Ns] = o[r];
    }
}

/* In-place transform of buf (n) using work (n). */
static void fft_1d(const fft_plan *p, cpx *buf, cpx *work, int sign)
{
    cpx *x = buf, *y = work;
    int Ns = 1;
    for (int s = 0; s < p->nstages; s++) {
        fft_pass(p, x, y, p->radix[s], Ns, sign);
        Ns *= p->radix[s];
        cpx *t = x; x = y; y = t;
    }
    if (x != buf)
        memcpy(buf, x, sizeof(cpx) * p->n);
}

/* 2-D transform of an H x W row-major complex plane. */
static void fft_2d(const fft_plan *ph, const fft_plan *pw, cpx *a, int H, int W, cpx *col, cpx *work, int sign)
{
    for (int y = 0; y < H; y++)
        fft_1d(pw, a + (size_t)y * W, work, sign);
    for (int x = 0; x < W; x++) {
        for (int y = 0; y < H; y++) col[y] = a[(size_t)y * W + x];
        fft_1d(ph, col, work, sign);
        for (int y = 0; y < H; y++) a[(size_t)y * W + x] = col[y];
    }
}

/* ------------------------------------------------------------ helpers */
static int clamp_idx(int i, int n, int border)
{
    if (i < n) return i;
    if (i < n + border) return n - 1;
    return 0;
}

static int align_up(int a, int b) { return (a % b != 0) ? (a - a % b + b) : a; }

static int max_prime_factor(int n)
{
    int best = 1;
    for (int f = 2; n > 1; f++)
        while (n % f == 0) { best = f; n /= f; }
    return best;
}

int fmvdcpu_snap(int n)
{
    n = align_up(n, 16);
    int hibit = 31;
    while (hibit >= 0 && !(n & (1u << hibit))) hibit--;
    if ((1u << hibit) == (unsigned)n) return n;
    unsigned hi = 1u << (hibit + 1);
    if (hi <= 1024) return (int)hi;
    return align_up(n, 512);
}

/* Kernel spectrum (full H x W complex, scaled by 1/(H W)) of a kH x kW
 * kernel centred at (kH/2, kW/2) -> (0, 0). */
static void kernel_spectrum(const float *k, int kH, int kW, int H, int W, const fft_plan *ph, const fft_plan *pw,
                            cpx *out, cpx *col, cpx *work)
{
    memset(out, 0, sizeof(cpx) * (size_t)H * W);
    for (int y = 0; y < kH; y++)
        for (int x = 0; x < kW; x++) {
            int yy = (y - kH / 2 + H) % H, xx = (x - kW / 2 + W) % W;
            out[(size_t)yy * W + xx].re = k[y * kW + x];
        }
    fft_2d(ph, pw, out, H, W, col, work, -1);
    float s = 1.0f / ((float)H * (float)W);
    for (size_t i = 0; i < (size_t)H * W; i++) { out[i].re *= s; out[i].im *= s; }
}

/* ---------------------------------------------------------------- API */
/* views:    V x D x dataH x dataW samples (bits 8 or 16)
 * weights:  V x dataH x dataW raw weights
 * k1, k2:   V x kH x kW normalised kernels (kernel 1, and the derived kernel 2)
 * out:      D x dataH x dataW samples
 * est:      optional D x fftH x fftW float estimates
 * Returns 0, or -1 if an FFT size has a prime factor above 31. */
int fmvdcpu_deconvolve(int bits, const void *views, const float *weights, const float *k1, const float *k2,
                       int V, int D, int dataH, int dataW, int kH, int kW, int iterations,
                       void *out, float *est, int nthreads)
{
    int H = fmvdcpu_snap(dataH + kH - 1);
    int W = fmvdcpu_snap(dataW + kW - 1);
    if (max_prime_factor(H) > 31 || max_prime_factor(W) > 31)
        return -1;
    size_t N = (size_t)H * W, dN = (size_t)dataH * dataW;
    fft_plan ph, pw;
    fft_plan_init(&ph, H);
    fft_plan_init(&pw, W);

    cpx *K = (cpx *)malloc(sizeof(cpx) * N * V), *Kh = (cpx *)malloc(sizeof(cpx) * N * V);
    {
        cpx *col = (cpx *)malloc(sizeof(cpx) * (H > W ? H : W));
        cpx *work = (cpx *)malloc(sizeof(cpx) * (H > W ? H : W));
        for (int v = 0; v < V; v++) {
            kernel_spectrum(k1 + (size_t)v * kH * kW, kH, kW, H, W, &ph, &pw, K + N * v, col, work);
            kernel_spectrum(k2 + (size_t)v * kH * kW, kH, kW, H, W, &ph, &pw, Kh + N * v, col, work);
        }
        free(col); free(work);
    }
    /* padded, normalised weights (borders kH/2 rows, kW/2 columns) */
    float *Wp = (float *)malloc(sizeof(float) * N * V), *Ws = (float *)calloc(N, sizeof(float));
    for (int v = 0; v < V; v++)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                float w = weights[(size_t)v * dN + (size_t)clamp_idx(y, dataH, kH / 2) * dataW + clamp_idx(x, dataW, kW / 2)];
                Wp[N * v + (size_t)y * W + x] = w;
                Ws[(size_t)y * W + x] += w;
            }
    for (int v = 0; v < V; v++)
        for (size_t i = 0; i < N; i++)
            if (Ws[i] > 0) Wp[N * v + i] /= Ws[i];

    int npairs = (D + 1) / 2;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
    {
        cpx *e = (cpx *)malloc(sizeof(cpx) * N), *c = (cpx *)malloc(sizeof(cpx) * N);
        cpx *col = (cpx *)malloc(sizeof(cpx) * (H > W ? H : W)), *work = (cpx *)malloc(sizeof(cpx) * (H > W ? H : W));
        float *dpad = (float *)malloc(sizeof(float) * N * 2 * V);
#pragma omp for schedule(dynamic, 1)
        for (int p = 0; p < npairs; p++) {
            int z0 = 2 * p, z1 = 2 * p + 1;
            int has1 = z1 < D;
            for (size_t i = 0; i < N; i++) { e[i].re = 10.0f * V; e[i].im = has1 ? 10.0f * V : 0.f; }
            /* padded data of the two planes (row border kW/2, column border kH/2) */
            for (int v = 0; v < V; v++)
                    for (int y = 0; y < H; y++)
                        for (int x = 0; x < W; x++) {
                            size_t src = (size_t)clamp_idx(y, dataH, kW / 2) * dataW + clamp_idx(x, dataW, kH / 2);
                            float a, b = 0.f;
                            if (bits == 16) {
                                const uint16_t *s = (const uint16_t *)views;
                                a = s[((size_t)v * D + z0) * dN + src];
                                if (has1) b = s[((size_t)v * D + z1) * dN + src];
                            } else {
                                const uint8_t *s = (const uint8_t *)views;
                                a = s[((size_t)v * D + z0) * dN + src];
                                if (has1) b = s[((size_t)v * D + z1) * dN + src];
                            }
                            dpad[2 * (N * v + (size_t)y * W + x)] = a;
                            dpad[2 * (N * v + (size_t)y * W + x) + 1] = b;
                        }
            for (int it = 0; it < iterations; it++)
                for (int v = 0; v < V; v++) {
                    const float *dv = dpad + 2 * N * v;
                    memcpy(c, e, sizeof(cpx) * N);
                    fft_2d(&ph, &pw, c, H, W, col, work, -1);
                    const cpx *kv = K + N * v;
                    for (size_t i = 0; i < N; i++) {
                        cpx a = c[i], k = kv[i];
                        c[i].re = a.re * k.re - a.im * k.im;
                        c[i].im = a.re * k.im + a.im * k.re;
                    }
                    fft_2d(&ph, &pw, c, H, W, col, work, +1);
                    for (size_t i = 0; i < N; i++) {
                        if (c[i].re > 1.f) c[i].re = dv[2 * i] / c[i].re;
                        if (c[i].im > 1.f) c[i].im = dv[2 * i + 1] / c[i].im;
                    }
                    fft_2d(&ph, &pw, c, H, W, col, work, -1);
                    const cpx *khv = Kh + N * v;
                    for (size_t i = 0; i < N; i++) {
                        cpx a = c[i], k = khv[i];
                        c[i].re = a.re * k.re - a.im * k.im;
                        c[i].im = a.re * k.im + a.im * k.re;
                    }
                    fft_2d(&ph, &pw, c, H, W, col, work, +1);
                    const float *wv = Wp + N * v;
                    for (size_t i = 0; i < N; i++) {
                        e[i].re += wv[i] * (e[i].re * c[i].re - e[i].re);
                        e[i].im += wv[i] * (e[i].im * c[i].im - e[i].im);
                    }
                }
            float maxv = (float)((1 << bits) - 1);
            for (int q = 0; q < 2; q++) {
                int z = q ? z1 : z0;
                if (z >= D) break;
                for (int y = 0; y < dataH; y++)
                    for (int x = 0; x < dataW; x++) {
                        float val = q ? e[(size_t)y * W + x].im : e[(size_t)y * W + x].re;
                        if (val > maxv) val = maxv;
                        if (val < 0.f) val = 0.f;
                        if (bits == 16) ((uint16_t *)out)[(size_t)z * dN + (size_t)y * dataW + x] = (uint16_t)val;
                        else ((uint8_t *)out)[(size_t)z * dN + (size_t)y * dataW + x] = (uint8_t)val;
                    }
                if (est)
                    for (size_t i = 0; i < N; i++) est[(size_t)z * N + i] = q ? e[i].im : e[i].re;
            }
        }
        free(e); free(c); free(col); free(work); free(dpad);
    }
    free(K); free(Kh); free(Wp); free(Ws);
    fft_plan_free(&ph);
    fft_plan_free(&pw);
    return 0;
}

int fmvdcpu_max_threads(void) { return omp_get_max_threads(); }
