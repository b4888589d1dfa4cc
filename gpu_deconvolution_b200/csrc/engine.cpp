// Plan-time preparation and the launch sequence of the RL engine.
//
// Plan time follows fmvd_initialize_cuda_* of the reference
// (fmvd_deconvolve.impl.cpp:130-203): FFT sizes by snapTransformSize,
// kernel 2 derived from the unnormalised kernels (fmvd_deconvolve.cpp:139-204),
// then the caller's kernels normalised in place (fmvd_deconvolve.impl.cpp:63-64),
// kernel spectra, and weights normalised over views
// (fmvd_deconvolve.impl.cpp:86-124).  Spectra are computed on the device by a
// direct separable DFT in FP32 with compensated sums; the small same-size
// convolutions of the compound kernels run on the device in FP32 too.  (FP64
// on the GPU is used only by the convergence statistics.)
#include "fmvd_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

namespace fmvd {

namespace {

// fmvd_deconvolve.cpp:53-68: double sum, float division.
void normalize_kernel(float *k, int n)
{
    double sum = 0;
    for (int i = 0; i < n; i++)
        sum += k[i];
    const float s = (float)sum;
    for (int i = 0; i < n; i++)
        k[i] /= s;
}

// fmvd_deconvolve.cpp:70-79: point mirror of a kw x kh kernel.
void invert_kernel(const float *k, float *out, int kw, int kh)
{
    for (int y = 0; y < kh; y++)
        for (int x = 0; x < kw; x++)
            out[y * kw + x] = k[(kh - y - 1) * kw + (kw - x - 1)];
}

// Clamp-padded circular convolution of a kernel-sized image on the device in
// FP32 (the reference's convolve_single_plane, fmvd_deconvolve.cpp:90-137,
// an FP32 cuFFT convolution).
bool conv_same(float *img, const float *k, int kw, int kh, float *d_a, float *d_b, float *d_c)
{
    const size_t bytes = sizeof(float) * kw * kh;
    if (!FMVD_CHECK(cudaMemcpy(d_a, img, bytes, cudaMemcpyHostToDevice)) ||
        !FMVD_CHECK(cudaMemcpy(d_b, k, bytes, cudaMemcpyHostToDevice)))
        return false;
    rl_conv_same(d_a, kh, kw, d_b, kh, kw, d_c, 0);
    return FMVD_CHECK(cudaGetLastError()) && FMVD_CHECK(cudaMemcpy(img, d_c, bytes, cudaMemcpyDeviceToHost));
}

// fmvd_deconvolve.cpp:139-204
bool compute_kernel2(float *const *k, int kw, int kh, int V, int type, std::vector<std::vector<float>> &k2)
{
    const int n = kw * kh;
    k2.assign(V, std::vector<float>(n));
    std::vector<float> t1(n), t2(n);
    float *d_a = nullptr, *d_b = nullptr, *d_c = nullptr;
    bool need_conv = (type == efficient_bayesian || type == optimization_1) && V > 1;
    if (need_conv) {
        if (!FMVD_CHECK(cudaMalloc(&d_a, n * sizeof(float))) || !FMVD_CHECK(cudaMalloc(&d_b, n * sizeof(float))) ||
            !FMVD_CHECK(cudaMalloc(&d_c, n * sizeof(float)))) {
            cudaFree(d_a);
            cudaFree(d_b);
            return false;
        }
    }
    bool ok = true;
    for (int v = 0; v < V && ok; v++) {
        float *out = k2[v].data();
        switch (type) {
        case independent:
            invert_kernel(k[v], out, kw, kh);
            break;
        case efficient_bayesian:
            invert_kernel(k[v], out, kw, kh);
            for (int w = 0; w < V && ok; w++) {
                if (w == v)
                    continue;
                invert_kernel(k[v], t1.data(), kw, kh);
                ok = conv_same(t1.data(), k[w], kw, kh, d_a, d_b, d_c);
                invert_kernel(k[w], t2.data(), kw, kh);
                ok = ok && conv_same(t1.data(), t2.data(), kw, kh, d_a, d_b, d_c);
                for (int i = 0; i < n; i++)
                    out[i] *= t1[i];
            }
            break;
        case optimization_1:
            invert_kernel(k[v], out, kw, kh);
            for (int w = 0; w < V && ok; w++) {
                if (w == v)
                    continue;
                invert_kernel(k[v], t1.data(), kw, kh);
                ok = conv_same(t1.data(), k[w], kw, kh, d_a, d_b, d_c);
                for (int i = 0; i < n; i++)
                    out[i] *= t1[i];
            }
            break;
        case optimization_2: {
            std::vector<float> e(n);
            for (int i = 0; i < n; i++)
                e[i] = (float)pow((double)k[v][i], (double)V);
            invert_kernel(e.data(), out, kw, kh);
            break;
        }
        default:
            report_error("fmvd: unknown psf type");
            ok = false;
        }
        if (ok)
            normalize_kernel(out, n);
    }
    cudaFree(d_a);
    cudaFree(d_b);
    cudaFree(d_c);
    return ok;
}

std::vector<double2> twiddles_d(int n)
{
    std::vector<double2> t(n);
    for (int i = 0; i < n; i++) {
        const double a = -2.0 * M_PI * (double)i / (double)n;
        t[i] = make_double2(cos(a), sin(a));
    }
    return t;
}

// Twiddle table of the warp FFT's four-step split N = T x E (zeros when N
// has no warp split), rl_warp_twiddle_entries(N) entries: with
// R8 = min(E, kWarpTwiddleRun) and J = E / R8,
//   [j * T + t] = exp(-2 pi i R8 j t / N) for j < J, t < T
//   [J * T + t] = exp(-2 pi i t / N)
std::vector<float2> warp_twiddles(int n)
{
    if (n > 1024)
        return warp_twiddles(kLineM);  // lines above 1024 run 512-point sub-transforms
    std::vector<float2> t(rl_warp_twiddle_entries(n), make_float2(0.f, 0.f));
    const int T = rl_warp_lanes(n);
    if (T == 0)
        return t;
    const int E = n / T;
    const int R8 = E < kWarpTwiddleRun ? E : kWarpTwiddleRun;
    const int J = E / R8;
    auto w = [n](long long k) {
        const double a = -2.0 * M_PI * (double)(k % n) / (double)n;
        return make_float2((float)cos(a), (float)sin(a));
    };
    for (int j = 0; j < J; j++)
        for (int l = 0; l < T; l++)
            t[j * T + l] = w((long long)R8 * j * l);
    for (int l = 0; l < T; l++)
        t[J * T + l] = w(l);
    return t;
}

} // namespace

int default_pairs_cap(int H, int W, int lanes)
{
    // Keep the complex work planes of the batches in flight (one per lane)
    // around 48 MB in total so that they stay resident in the 126 MB L2
    // between passes.
    const size_t per_pair = (size_t)H * W * sizeof(float2);
    size_t cap = ((size_t)48 << 20) / per_pair / (size_t)(lanes > 1 ? lanes : 1);
    if (cap < 1)
        cap = 1;
    if (cap > 64)
        cap = 64;
    return (int)cap;
}

Engine *engine_create(int bits, int dataH, int dataW, const float *const *h_Weights, float **h_Kernel, int kH,
                      int kW, int psf_type, int nViews, int pairs_cap, int col_warps, int lanes)
{
    if (bits != 8 && bits != 16) {
        report_error("fmvd: unsupported sample size");
        return nullptr;
    }
    if (dataH < 1 || dataW < 1 || kH < 1 || kW < 1 || nViews < 1 || !h_Weights || !h_Kernel) {
        report_error("fmvd: invalid plan arguments");
        return nullptr;
    }
    const int H = snap_transform_size(dataH + kH - 1);
    const int W = snap_transform_size(dataW + kW - 1);
    if (!rl_length_supported(H) || !rl_length_supported(W)) {
        char msg[160];
        snprintf(msg, sizeof(msg), "fmvd: padded plane %d x %d is not supported (each side must be <= 4096)", H, W);
        report_error(msg);
        return nullptr;
    }
    const int cw = rl_col_warps(H, W, col_warps);
    if (cw < 0) {
        char msg[160];
        snprintf(msg, sizeof(msg), "fmvd: %d column-pass warps do not fit a %d x %d plane", col_warps, H, W);
        report_error(msg);
        return nullptr;
    }
    int dev = 0;
    if (!FMVD_CHECK(cudaGetDevice(&dev)))
        return nullptr;

    Engine *e = new Engine();
    memset(e, 0, sizeof(Engine));
    e->dims.H = H;
    e->dims.W = W;
    e->dims.dataH = dataH;
    e->dims.dataW = dataW;
    e->dims.V = nViews;
    e->dims.bits = bits;
    e->dims.byD = kW / 2;  // fmvd_deconvolve_cuda.impl.cu:76-77 receives (kernelH, kernelW) swapped
    e->dims.bxD = kH / 2;
    e->dims.byW = kH / 2;
    e->dims.bxW = kW / 2;
    e->dims.col_warps = cw;
    e->dims.radix_step = kRadixDft;
    e->kH = kH;
    e->kW = kW;
    e->device = dev;
    e->lanes = lanes < 1 ? 1 : (lanes > kMaxLanes ? kMaxLanes : lanes);
    e->pairs_cap = pairs_cap > 0 ? pairs_cap : default_pairs_cap(H, W, e->lanes);
    e->spec_elems = rl_spectrum_elems(H, W);

    // kernel 2 from the unnormalised kernels, then normalise the caller's kernels
    std::vector<std::vector<float>> k2;
    if (!compute_kernel2(h_Kernel, kW, kH, nViews, psf_type, k2)) {
        engine_destroy(e);
        return nullptr;
    }
    for (int v = 0; v < nViews; v++)
        normalize_kernel(h_Kernel[v], kW * kH);

    const size_t plane = (size_t)dataH * dataW;
    bool ok = FMVD_CHECK(cudaMalloc(&e->spec, sizeof(float2) * e->spec_elems * 2 * nViews)) &&
              FMVD_CHECK(cudaMalloc(&e->weights, sizeof(float) * plane * nViews)) &&
              FMVD_CHECK(cudaMalloc(&e->C, sizeof(float2) * (size_t)H * W * e->pairs_cap)) &&
              FMVD_CHECK(cudaMalloc(&e->est, sizeof(float2) * (size_t)H * W * e->pairs_cap)) &&
              FMVD_CHECK(cudaMalloc(&e->twH, sizeof(float2) * H)) && FMVD_CHECK(cudaMalloc(&e->twW, sizeof(float2) * W)) &&
              FMVD_CHECK(cudaMalloc(&e->wtwH, sizeof(float2) * rl_warp_twiddle_entries(H))) &&
              FMVD_CHECK(cudaMalloc(&e->wtwW, sizeof(float2) * rl_warp_twiddle_entries(W))) &&
              FMVD_CHECK(cudaMalloc(&e->status, sizeof(int))) && FMVD_CHECK(cudaMemset(e->status, 0, sizeof(int)));
    if (ok && e->lanes > 1)
        ok = FMVD_CHECK(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
    for (int l = 0; ok && l + 1 < e->lanes; l++)
        ok = FMVD_CHECK(cudaMalloc(&e->laneC[l], sizeof(float2) * (size_t)H * W * e->pairs_cap)) &&
             FMVD_CHECK(cudaMalloc(&e->laneEst[l], sizeof(float2) * (size_t)H * W * e->pairs_cap)) &&
             FMVD_CHECK(cudaStreamCreateWithFlags(&e->side[l], cudaStreamNonBlocking)) &&
             FMVD_CHECK(cudaEventCreateWithFlags(&e->ev_join[l], cudaEventDisableTiming));
    if (!ok) {
        engine_destroy(e);
        return nullptr;
    }

    // twiddle tables
    {
        std::vector<double2> tH = twiddles_d(H), tW = twiddles_d(W);
        std::vector<float2> fH(H), fW(W);
        for (int i = 0; i < H; i++)
            fH[i] = make_float2((float)tH[i].x, (float)tH[i].y);
        for (int i = 0; i < W; i++)
            fW[i] = make_float2((float)tW[i].x, (float)tW[i].y);
        std::vector<float2> wH = warp_twiddles(H), wW = warp_twiddles(W);
        ok = FMVD_CHECK(cudaMemcpy(e->twH, fH.data(), sizeof(float2) * H, cudaMemcpyHostToDevice)) &&
             FMVD_CHECK(cudaMemcpy(e->twW, fW.data(), sizeof(float2) * W, cudaMemcpyHostToDevice)) &&
             FMVD_CHECK(cudaMemcpy(e->wtwH, wH.data(), sizeof(float2) * wH.size(), cudaMemcpyHostToDevice)) &&
             FMVD_CHECK(cudaMemcpy(e->wtwW, wW.data(), sizeof(float2) * wW.size(), cudaMemcpyHostToDevice));

        // kernel spectra (FP32 on the device; the twiddle tables are the
        // float tables above, computed in double on the host and rounded)
        float2 *work = nullptr;
        float *d_k = nullptr;
        ok = ok && FMVD_CHECK(cudaMalloc(&work, sizeof(float2) * ((size_t)H * W + (size_t)kH * W))) &&
             FMVD_CHECK(cudaMalloc(&d_k, sizeof(float) * kH * kW));
        for (int v = 0; v < nViews && ok; v++) {
            for (int which = 0; which < 2 && ok; which++) {
                const float *src = which == 0 ? h_Kernel[v] : k2[v].data();
                ok = FMVD_CHECK(cudaMemcpy(d_k, src, sizeof(float) * kH * kW, cudaMemcpyHostToDevice));
                if (ok) {
                    rl_kernel_spectrum(d_k, kH, kW, H, W, e->twH, e->twW, work,
                                       e->spec + e->spec_elems * (2 * v + which), e->dims.col_warps, 0);
                    ok = FMVD_CHECK(cudaGetLastError()) && FMVD_CHECK(cudaDeviceSynchronize());
                }
            }
        }
        cudaFree(work);
        cudaFree(d_k);
    }

    // weights normalised over views
    if (ok) {
        float *raw = nullptr;
        ok = FMVD_CHECK(cudaMalloc(&raw, sizeof(float) * plane * nViews));
        for (int v = 0; v < nViews && ok; v++)
            ok = FMVD_CHECK(cudaMemcpy(raw + plane * v, h_Weights[v], sizeof(float) * plane, cudaMemcpyHostToDevice));
        if (ok) {
            rl_normalize_weights(raw, e->weights, nViews, plane, 0);
            ok = FMVD_CHECK(cudaGetLastError()) && FMVD_CHECK(cudaDeviceSynchronize());
        }
        cudaFree(raw);
    }
    if (!ok) {
        engine_destroy(e);
        return nullptr;
    }
    return e;
}

void engine_destroy(Engine *e)
{
    if (!e)
        return;
    cudaFree(e->spec);
    cudaFree(e->weights);
    cudaFree(e->C);
    cudaFree(e->est);
    cudaFree(e->twH);
    cudaFree(e->twW);
    cudaFree(e->wtwH);
    cudaFree(e->wtwW);
    cudaFree(e->status);
    for (int l = 0; l + 1 < kMaxLanes; l++) {
        cudaFree(e->laneC[l]);
        cudaFree(e->laneEst[l]);
        if (e->side[l])
            cudaStreamDestroy(e->side[l]);
        if (e->ev_join[l])
            cudaEventDestroy(e->ev_join[l]);
    }
    if (e->ev_fork)
        cudaEventDestroy(e->ev_fork);
    delete e;
}

void engine_batch(Engine *e, const void *data, size_t view_stride, void *out, int nplanes, int iterations,
                  cudaStream_t s, const float *init)
{
    const int V = e->dims.V;
    RlBatch b;
    b.C = e->C;
    b.est = e->est;
    b.data = data;
    b.view_stride = view_stride;
    b.plane_stride = (size_t)e->dims.dataH * e->dims.dataW;
    b.weights = e->weights;
    b.out = out;
    b.npairs = (nplanes + 1) / 2;
    b.nplanes = nplanes;
    b.init_value = 10.0f * (float)V;  // fmvd_deconvolve_cuda.impl.cu:62, once per view
    b.init = init;
    b.status = e->status;
    RlTables t{e->twH, e->twW, e->wtwH, e->wtwW};
    const float2 *spec = e->spec;
    const size_t se = e->spec_elems;

    rl_init(e->dims, b, t, s);
    if (iterations <= 0) {
        rl_write_estimate(e->dims, b, s);
        return;
    }
    rl_col(e->dims, b, t, spec + se * 0, s);
    for (int it = 0; it < iterations; it++) {
        for (int v = 0; v < V; v++) {
            const bool last = (it == iterations - 1) && (v == V - 1);
            rl_divide(e->dims, b, t, v, s);
            rl_col(e->dims, b, t, spec + se * (2 * v + 1), s);
            rl_update(e->dims, b, t, v, last, s);
            if (!last)
                rl_col(e->dims, b, t, spec + se * (2 * ((v + 1) % V)), s);
        }
    }
}

bool engine_check_status(Engine *e)
{
    int st = 0;
    if (!FMVD_CHECK(cudaMemcpy(&st, e->status, sizeof(int), cudaMemcpyDeviceToHost)))
        return false;
    if (st) {
        cudaMemset(e->status, 0, sizeof(int));
        report_error("fmvd: a bulk copy into shared memory did not complete in time");
        return false;
    }
    return true;
}

bool engine_run(Engine *e, const void *data, size_t view_stride, void *out, int nplanes, int iterations,
                float *est_out, cudaStream_t s, const float *init)
{
    const size_t plane = (size_t)e->dims.dataH * e->dims.dataW;
    const size_t fplane = (size_t)e->dims.H * e->dims.W;
    const size_t es = e->dims.bits == 16 ? 2 : 1;
    const int per = 2 * e->pairs_cap;
    // more lanes only when there are several batches
    const int nbatches = (nplanes + per - 1) / per;
    const int used = e->lanes < nbatches ? e->lanes : nbatches;
    Engine lane_eng[kMaxLanes];
    cudaStream_t lane_s[kMaxLanes];
    lane_eng[0] = *e;
    lane_s[0] = s;
    if (used > 1 && !FMVD_CHECK(cudaEventRecord(e->ev_fork, s)))
        return false;
    for (int l = 1; l < used; l++) {
        lane_eng[l] = *e;
        lane_eng[l].C = e->laneC[l - 1];
        lane_eng[l].est = e->laneEst[l - 1];
        lane_s[l] = e->side[l - 1];
        if (!FMVD_CHECK(cudaStreamWaitEvent(lane_s[l], e->ev_fork, 0)))
            return false;
    }
    for (int z0 = 0, k = 0; z0 < nplanes; z0 += per, k++) {
        const int n = nplanes - z0 < per ? nplanes - z0 : per;
        Engine *lane = &lane_eng[k % used];
        const cudaStream_t ls = lane_s[k % used];
        engine_batch(lane, (const char *)data + z0 * plane * es, view_stride, (char *)out + z0 * plane * es, n,
                     iterations, ls, init ? init + (size_t)z0 * fplane : nullptr);
        if (est_out)
            rl_split_estimate(e->dims, lane->est, n, est_out + (size_t)z0 * fplane, ls);
        if (!FMVD_CHECK(cudaGetLastError()))
            return false;
    }
    for (int l = 1; l < used; l++)
        if (!FMVD_CHECK(cudaEventRecord(e->ev_join[l - 1], lane_s[l])) ||
            !FMVD_CHECK(cudaStreamWaitEvent(s, e->ev_join[l - 1], 0)))
            return false;
    return true;
}

} // namespace fmvd
