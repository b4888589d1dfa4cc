// Host-buffer reconstruction: resampling of every view into the common frame
// followed by plain RL, from source volumes in host memory to the result in
// host memory, with the resampled frame kept on the device.
//
// The reference's plugin path moves the resampled frame through the host
// twice (transform_cuda_* writes it out, fmvd_deconvolve_planes_cuda_* reads
// it back plane by plane).  Here the host traffic is the source volumes in and
// the result out: the sources are uploaded once (on a copy stream, view by
// view, the first chunk starting on each view as it lands), then target
// planes are processed in chunks: a resampling stream fills a device chunk
// with the V views' planes (double-buffered, so chunk k + 1 is resampled
// while chunk k deconvolves), the compute stream deconvolves it and writes
// the chunk's samples, the copy stream moves the previous chunk's result to
// pinned staging and the host thread moves it into the caller's buffer (with
// a few helper threads: one thread copies only a few GB/s).
#include "fmvd_b200.h"
#include "fmvd_internal.h"
#include "transform_kernels.h"

#include <string.h>
#include <vector>

struct fmvd_b200_reconstructor {
    fmvd_b200_plan *plan;
    int V, w, h, d, tw, th, td, chunk, bits;
    size_t pitch, es;
    void *src = nullptr;          // V x d x h x pitch samples
    void *frame[2] = {};          // V x chunk x th x tw samples
    void *out[2] = {};            // chunk x th x tw samples
    void *stage[2] = {};          // pinned, chunk x th x tw samples
    int *status = nullptr;
    cudaStream_t comp = nullptr, copy = nullptr, rs = nullptr;
    cudaEvent_t done[2] = {}, copied[2] = {}, resampled[2] = {};
    std::vector<cudaEvent_t> uploaded;  // per view: its source volume is on the device
};

namespace {

void release(fmvd_b200_reconstructor *r)
{
    if (!r)
        return;
    cudaFree(r->src);
    for (int i = 0; i < 2; i++) {
        cudaFree(r->frame[i]);
        cudaFree(r->out[i]);
        cudaFreeHost(r->stage[i]);
        if (r->done[i])
            cudaEventDestroy(r->done[i]);
        if (r->copied[i])
            cudaEventDestroy(r->copied[i]);
        if (r->resampled[i])
            cudaEventDestroy(r->resampled[i]);
    }
    for (cudaEvent_t e : r->uploaded)
        if (e)
            cudaEventDestroy(e);
    cudaFree(r->status);
    if (r->comp)
        cudaStreamDestroy(r->comp);
    if (r->copy)
        cudaStreamDestroy(r->copy);
    if (r->rs)
        cudaStreamDestroy(r->rs);
    delete r;
}

} // namespace

extern "C" {

fmvd_b200_reconstructor *fmvd_b200_reconstructor_create(fmvd_b200_plan *plan, int views, int w, int h, int d,
                                                        int tw, int th, int td, int chunk_planes)
{
    if (!plan || views < 1 || views != plan->eng->dims.V || w < 1 || h < 1 || d < 1 || td < 1 ||
        tw != plan->eng->dims.dataW || th != plan->eng->dims.dataH) {
        fmvd::report_error("fmvd: fmvd_b200_reconstructor_create: the plan's views and plane size must match the "
                           "frame");
        return nullptr;
    }
    auto *r = new fmvd_b200_reconstructor();
    r->plan = plan;
    r->V = views;
    r->w = w;
    r->h = h;
    r->d = d;
    r->tw = tw;
    r->th = th;
    r->td = td;
    r->bits = plan->eng->dims.bits;
    r->es = r->bits == 16 ? 2 : 1;
    r->pitch = fmvd::source_pitch(r->bits, w);
    const int batch = 2 * plan->eng->pairs_cap;
    int chunk = chunk_planes > 0 ? chunk_planes : 8 * batch;
    if (chunk > td)
        chunk = td;
    r->chunk = chunk;
    const size_t plane = (size_t)tw * th * r->es;
    bool ok = FMVD_CHECK(cudaMalloc(&r->src, (size_t)views * d * h * r->pitch * r->es)) &&
              FMVD_CHECK(cudaMalloc(&r->status, sizeof(int))) && FMVD_CHECK(cudaMemset(r->status, 0, sizeof(int))) &&
              FMVD_CHECK(cudaStreamCreateWithFlags(&r->comp, cudaStreamNonBlocking)) &&
              FMVD_CHECK(cudaStreamCreateWithFlags(&r->copy, cudaStreamNonBlocking)) &&
              FMVD_CHECK(cudaStreamCreateWithFlags(&r->rs, cudaStreamNonBlocking));
    for (int i = 0; i < 2 && ok; i++)
        ok = FMVD_CHECK(cudaMalloc(&r->frame[i], (size_t)views * chunk * plane)) &&
             FMVD_CHECK(cudaMalloc(&r->out[i], (size_t)chunk * plane)) &&
             FMVD_CHECK(cudaMallocHost(&r->stage[i], (size_t)chunk * plane)) &&
             FMVD_CHECK(cudaEventCreateWithFlags(&r->done[i], cudaEventDisableTiming)) &&
             FMVD_CHECK(cudaEventCreateWithFlags(&r->copied[i], cudaEventDisableTiming)) &&
             FMVD_CHECK(cudaEventCreateWithFlags(&r->resampled[i], cudaEventDisableTiming));
    r->uploaded.assign(views, nullptr);
    for (int v = 0; v < views && ok; v++)
        ok = FMVD_CHECK(cudaEventCreateWithFlags(&r->uploaded[v], cudaEventDisableTiming));
    if (!ok) {
        release(r);
        return nullptr;
    }
    return r;
}

int fmvd_b200_reconstruct_host(fmvd_b200_reconstructor *r, const void *const *h_views, const float *h_inverses,
                               int iterations, void *h_out)
{
    if (!r || !h_views || !h_inverses || !h_out) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_reconstruct_host");
        return 1;
    }
    const size_t es = r->es;
    const size_t plane = (size_t)r->tw * r->th * es;
    const size_t vol = (size_t)r->d * r->h * r->pitch * es;
    bool ok = FMVD_CHECK(cudaMemsetAsync(r->status, 0, sizeof(int), r->rs));
    // sources: each view d x h x w contiguous on the host -> pitched device
    // rows, on the copy stream; the first chunk resamples view v as soon as
    // view v has landed, so the upload of later views overlaps it
    for (int v = 0; v < r->V && ok; v++)
        ok = FMVD_CHECK(cudaMemcpy2DAsync((char *)r->src + v * vol, r->pitch * es, h_views[v], (size_t)r->w * es,
                                          (size_t)r->w * es, (size_t)r->h * r->d, cudaMemcpyHostToDevice, r->copy)) &&
             FMVD_CHECK(cudaEventRecord(r->uploaded[v], r->copy));
    const int nchunks = (r->td + r->chunk - 1) / r->chunk;
    auto planes_of = [&](int k) { return r->td - k * r->chunk < r->chunk ? r->td - k * r->chunk : r->chunk; };
    for (int k = 0; k < nchunks && ok; k++) {
        const int b = k & 1, z0 = k * r->chunk, n = planes_of(k);
        if (k >= 2)  // the deconvolution of chunk k - 2 has read frame[b]
            ok = FMVD_CHECK(cudaStreamWaitEvent(r->rs, r->done[b], 0));
        for (int v = 0; v < r->V && ok; v++)
            ok = (k > 0 || FMVD_CHECK(cudaStreamWaitEvent(r->rs, r->uploaded[v], 0))) &&
                 fmvd::resample_device(r->bits, (const char *)r->src + v * vol, r->pitch, r->w, r->h, r->d, r->tw,
                                       r->th, z0, n, h_inverses + 12 * v,
                                       (char *)r->frame[b] + (size_t)v * r->chunk * plane, nullptr, r->status,
                                       r->rs);
        ok = ok && FMVD_CHECK(cudaEventRecord(r->resampled[b], r->rs));
        if (ok && k >= 2)  // the copy of chunk k - 2 has read out[b]
            ok = FMVD_CHECK(cudaStreamWaitEvent(r->comp, r->copied[b], 0));
        ok = ok && FMVD_CHECK(cudaStreamWaitEvent(r->comp, r->resampled[b], 0)) &&
             fmvd::engine_run(r->plan->eng, r->frame[b], (size_t)r->chunk * r->tw * r->th, r->out[b], n,
                                    iterations, nullptr, r->comp) &&
             FMVD_CHECK(cudaEventRecord(r->done[b], r->comp)) &&
             FMVD_CHECK(cudaStreamWaitEvent(r->copy, r->done[b], 0)) &&
             FMVD_CHECK(cudaMemcpyAsync(r->stage[b], r->out[b], n * plane, cudaMemcpyDeviceToHost, r->copy)) &&
             FMVD_CHECK(cudaEventRecord(r->copied[b], r->copy));
        if (ok && k >= 1) {  // previous chunk: staging -> caller's buffer while this chunk computes
            const int pb = (k - 1) & 1;
            ok = FMVD_CHECK(cudaEventSynchronize(r->copied[pb]));
            if (ok)
                fmvd::host_copy((char *)h_out + (size_t)(k - 1) * r->chunk * plane, r->stage[pb],
                                planes_of(k - 1) * plane);
        }
    }
    if (ok) {
        const int k = nchunks - 1, b = k & 1;
        ok = FMVD_CHECK(cudaEventSynchronize(r->copied[b]));
        if (ok)
            fmvd::host_copy((char *)h_out + (size_t)k * r->chunk * plane, r->stage[b], planes_of(k) * plane);
    }
    int status = 0;
    // everything queued has finished before returning, also after a failure:
    // the copies read the caller's views
    const bool idle = FMVD_CHECK(cudaStreamSynchronize(r->rs)) & FMVD_CHECK(cudaStreamSynchronize(r->comp)) &
                      FMVD_CHECK(cudaStreamSynchronize(r->copy));
    ok = ok && idle && FMVD_CHECK(cudaMemcpy(&status, r->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (ok && status) {
        fmvd::report_error("fmvd: a resampler brick load did not complete in time");
        ok = false;
    }
    return ok && fmvd::engine_check_status(r->plan->eng) ? 0 : 1;
}

void fmvd_b200_reconstructor_destroy(fmvd_b200_reconstructor *r)
{
    if (!r)
        return;
    cudaStreamSynchronize(r->rs);
    cudaStreamSynchronize(r->comp);
    cudaStreamSynchronize(r->copy);
    release(r);
}

} // extern "C"
