// Test-infrastructure driver for the reference library built from the
// upstream sources (oracle/_ref/libfmvd_ref.so).  Only the tests, the golden
// fixture generator and bench.py's reference leg load it.
//
// It feeds the reference's public C API (fmvd_initialize_cuda_* /
// fmvd_deconvolve_planes_cuda_* / fmvd_destroy_cuda_*,
// fmvd_deconvolve.impl.cpp:130-336) from host arrays through the
// datasource/datasink callbacks, exactly as the reference's own file reader
// does (fmvd_deconvolve_hdd.impl.cpp:16-34).  With nstreams == 1 the sink runs
// right after cudaStreamSynchronize of the only stream
// (fmvd_deconvolve.impl.cpp:239-241), so plan->d_estimate then holds the float
// estimate of the plane being returned; the harness copies it out.
#include "fmvd_deconvolve.h"
#include "fmvd_cuda_utils.h"

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <stdio.h>

namespace {

struct Feed {
    const void *views;      // V x D x H x W samples
    void *out;              // (returned planes) x H x W samples
    float *est;             // (returned planes) x fftH x fftW floats, or null
    int V, D, H, W;
    int next, returned, max_returned;
    int source_calls;
    size_t sample_bytes;
    const void *plan;
    int fftH, fftW, nstreams;
};

Feed g_feed;
int g_error = 0;
char g_error_msg[512];

void record_error(void *, const char *msg)
{
    g_error = 1;
    snprintf(g_error_msg, sizeof(g_error_msg), "%s", msg);
}

template <typename S>
int source(S **buffer, int offset)
{
    g_feed.source_calls++;
    if (g_feed.next >= g_feed.D)
        return 0;
    size_t plane = (size_t)g_feed.H * g_feed.W;
    const S *views = (const S *)g_feed.views;
    for (int v = 0; v < g_feed.V; v++)
        memcpy(buffer[v] + offset, views + ((size_t)v * g_feed.D + g_feed.next) * plane, plane * sizeof(S));
    g_feed.next++;
    return 1;
}

template <typename S, typename P>
void sink(S *buffer)
{
    size_t plane = (size_t)g_feed.H * g_feed.W;
    if (g_feed.returned < g_feed.max_returned) {
        memcpy((S *)g_feed.out + (size_t)g_feed.returned * plane, buffer, plane * sizeof(S));
        if (g_feed.est && g_feed.nstreams == 1) {
            const P *plan = (const P *)g_feed.plan;
            size_t fplane = (size_t)plan->fftH * plan->fftW;
            cudaMemcpy(g_feed.est + (size_t)g_feed.returned * fplane, plan->d_estimate,
                       fplane * sizeof(float), cudaMemcpyDeviceToHost);
        }
    }
    g_feed.returned++;
}

int source16(unsigned short **b, int o) { return source<unsigned short>(b, o); }
int source8(unsigned char **b, int o) { return source<unsigned char>(b, o); }
void sink16(unsigned short *b) { sink<unsigned short, fmvd_plan_cuda_16>(b); }
void sink8(unsigned char *b) { sink<unsigned char, fmvd_plan_cuda_8>(b); }

} // namespace

extern "C" {

const char *ref_last_error(void) { return g_error ? g_error_msg : ""; }

// Deconvolve V x D x H x W views through the reference library.
// kernels: V x kH x kW floats (modified in place: the reference normalises
// the caller's kernels).  weights: V x H x W floats.
// out: room for max_returned planes.  est: room for max_returned float
// planes of fftH x fftW (only filled with nstreams == 1).  stats[0] = number of
// datasource calls, stats[1] = number of datasink calls, stats[2] = fftH,
// stats[3] = fftW.  Returns 0 on success.
int ref_deconvolve(int bits, const void *views, int V, int D, int H, int W,
                   const float *weights, float *kernels, int kH, int kW,
                   int psf_type, int iterations, int nstreams,
                   void *out, int max_returned, float *est, int *stats)
{
    g_error = 0;
    setErrorHandler(record_error, NULL);
    memset(&g_feed, 0, sizeof(g_feed));
    g_feed.views = views;
    g_feed.out = out;
    g_feed.est = est;
    g_feed.V = V; g_feed.D = D; g_feed.H = H; g_feed.W = W;
    g_feed.max_returned = max_returned;
    g_feed.nstreams = nstreams;

    const float **w = new const float *[V];
    float **k = new float *[V];
    for (int v = 0; v < V; v++) {
        w[v] = weights + (size_t)v * H * W;
        k[v] = kernels + (size_t)v * kH * kW;
    }
    if (bits == 16) {
        fmvd_plan_cuda_16 *plan = fmvd_initialize_cuda_16(H, W, w, k, kH, kW, (fmvd_psf_type)psf_type,
                                                          V, nstreams, source16, sink16);
        g_feed.plan = plan;
        stats[2] = plan->fftH; stats[3] = plan->fftW;
        fmvd_deconvolve_planes_cuda_16(plan, iterations);
        fmvd_destroy_cuda_16(plan);
    } else {
        fmvd_plan_cuda_8 *plan = fmvd_initialize_cuda_8(H, W, w, k, kH, kW, (fmvd_psf_type)psf_type,
                                                        V, nstreams, source8, sink8);
        g_feed.plan = plan;
        stats[2] = plan->fftH; stats[3] = plan->fftW;
        fmvd_deconvolve_planes_cuda_8(plan, iterations);
        fmvd_destroy_cuda_8(plan);
    }
    cudaDeviceSynchronize();
    stats[0] = g_feed.source_calls;
    stats[1] = g_feed.returned;
    delete[] w;
    delete[] k;
    return g_error;
}

// The reference's file-based entry (fmvd_deconvolve_hdd.impl.cpp:36-76),
// three streams, reading raw views and writing the raw result.
int ref_deconvolve_files(int bits, const char **view_paths, const char *out_path, int W, int H, int D,
                         float *weights, float *kernels, int kH, int kW, int psf_type, int V, int iterations)
{
    g_error = 0;
    setErrorHandler(record_error, NULL);
    FILE **files = new FILE *[V];
    float **w = new float *[V];
    float **k = new float *[V];
    for (int v = 0; v < V; v++) {
        files[v] = fopen(view_paths[v], "rb");
        if (!files[v])
            return -1;
        w[v] = weights + (size_t)v * H * W;
        k[v] = kernels + (size_t)v * kH * kW;
    }
    FILE *out = fopen(out_path, "wb");
    if (!out)
        return -1;
    if (bits == 16)
        fmvd_deconvolve_files_cuda_16(files, out, W, H, D, w, k, kH, kW, (fmvd_psf_type)psf_type, V, iterations);
    else
        fmvd_deconvolve_files_cuda_8(files, out, W, H, D, w, k, kH, kW, (fmvd_psf_type)psf_type, V, iterations);
    for (int v = 0; v < V; v++)
        fclose(files[v]);
    fclose(out);
    delete[] files;
    delete[] w;
    delete[] k;
    return g_error;
}

} // extern "C"
