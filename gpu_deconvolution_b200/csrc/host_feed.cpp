// A C caller of the drop-in streaming API over volumes held in host memory
// (built as lib/libfmvd_host_feed.so, linked against the main library).
//
// It is what a C or C++ program that used the reference library does: it
// creates a plan with fmvd_initialize_cuda_16 and hands fmvd_deconvolve_planes_
// cuda_16 a datasource that copies the next plane of every view into the
// plan's buffers and a datasink that copies each result plane out, the same
// shape as the reference's own file reader (fmvd_deconvolve_hdd.impl.cpp:
// 16-34) with memory instead of files.  The benchmark times the drop-in path
// through it, so that no interpreter sits inside the per-plane callbacks, and
// the tests use it to check the C-callback path end to end.
//
// Like the reference's file entry point, it keeps its callback state in
// file-scope variables: one call at a time per process.
#include "fmvd_deconvolve.h"

#include <string.h>
#include <vector>

namespace {

struct Feed {
    const unsigned short *views = nullptr;  // V x D x H x W
    unsigned short *out = nullptr;          // max_out x H x W
    int V = 0, D = 0, next = 0, returned = 0, max_out = 0;
    size_t plane = 0;
    int source_calls = 0;
};

Feed g_feed;

int feed_source(unsigned short **buffer, int offset)
{
    g_feed.source_calls++;
    if (g_feed.next >= g_feed.D)
        return 0;
    for (int v = 0; v < g_feed.V; v++)
        memcpy(buffer[v] + offset, g_feed.views + ((size_t)v * g_feed.D + g_feed.next) * g_feed.plane,
               g_feed.plane * sizeof(unsigned short));
    g_feed.next++;
    return 1;
}

void feed_sink(unsigned short *buffer)
{
    if (g_feed.returned < g_feed.max_out)
        memcpy(g_feed.out + (size_t)g_feed.returned * g_feed.plane, buffer, g_feed.plane * sizeof(unsigned short));
    g_feed.returned++;
}

} // namespace

extern "C" {

// Deconvolves V x D x dataH x dataW 16-bit views through fmvd_initialize /
// deconvolve_planes / destroy_cuda_16.  weights: V x dataH x dataW floats;
// kernels: V x kernelH x kernelW floats (normalised in place, as the API
// does).  out: room for max_out planes.  counts (optional): [0] datasource
// calls, [1] datasink calls.  Returns the number of planes the sink received,
// or -1 if the plan could not be created.
int fmvd_feed_deconvolve_16(const unsigned short *views, int V, int D, int dataH, int dataW, const float *weights,
                            float *kernels, int kernelH, int kernelW, int psf_type, int iterations, int nstreams,
                            unsigned short *out, int max_out, int *counts)
{
    g_feed = Feed();
    g_feed.views = views;
    g_feed.out = out;
    g_feed.V = V;
    g_feed.D = D;
    g_feed.max_out = max_out;
    g_feed.plane = (size_t)dataH * dataW;
    std::vector<const float *> w(V);
    std::vector<float *> k(V);
    for (int v = 0; v < V; v++) {
        w[v] = weights + (size_t)v * dataH * dataW;
        k[v] = kernels + (size_t)v * kernelH * kernelW;
    }
    fmvd_plan_cuda_16 *plan = fmvd_initialize_cuda_16(dataH, dataW, w.data(), k.data(), kernelH, kernelW,
                                                      (fmvd_psf_type)psf_type, V, nstreams, feed_source, feed_sink);
    if (!plan)
        return -1;
    fmvd_deconvolve_planes_cuda_16(plan, iterations);
    fmvd_destroy_cuda_16(plan);
    if (counts) {
        counts[0] = g_feed.source_calls;
        counts[1] = g_feed.returned;
    }
    return g_feed.returned;
}

} // extern "C"
