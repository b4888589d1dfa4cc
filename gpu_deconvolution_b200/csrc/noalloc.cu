// fmvd_b200_deconvolve_device_noalloc: the device-resident deconvolution of
// a plan with its work memory taken from a fixed array of this library, so the
// call itself allocates nothing.
//
// Why: fmvd_b200_deconvolve_device runs in the plan's own work planes (two
// complex planes per batched plane pair: 16 MiB per pair at 1024 x 1024, and
// the automatic batch holds several pairs), sized when the plan is created.
// A caller that keeps many plans alive at once (one per view configuration or
// plane size) and has no device memory to spare for each plan's full batch of
// work planes -- the rest of the GPU already holds its frame buffers, or
// another allocator has reserved it -- creates its plans with
// pairs_per_batch = 1 and deconvolves through this entry point, whose work
// planes live in one array shared by every plan and reserved when the
// library's module is loaded on a device.  Nothing here calls cudaMalloc,
// cudaFree or any routine that allocates.
//
// Limit: the array is kScratchBytes (64 MiB).  Its first 256 bytes hold the
// wait-status word; the rest holds the work planes of as many plane pairs as
// fit, at most the plan's own batch size.  A plan whose padded plane does not
// fit one pair (more than about 4.19 M complex points, e.g. 2048 x 2048) is
// rejected with an error.
//
// Sharing: every call on a device uses the same array, and the array keeps
// the last call's contents.  The status word is cleared at the start of each
// call; the work planes are written before they are read.  Calls that
// overlap in time on one device (from two host threads, or queued on two
// streams) race on the array and corrupt each other's results: serialise them.
#include "fmvd_b200.h"
#include "fmvd_internal.h"

#include <mutex>
#include <stdio.h>

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr size_t kStatusBytes = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_lock;
void *g_scratch_addr[kMaxDevices];

// Device address of g_scratch on the current device, looked up once per
// device (the first call on a device does this set-up; make that first call
// before any stream capture).  Null after reporting an error.
void *scratch_address()
{
    int dev = -1;
    if (!FMVD_CHECK(cudaGetDevice(&dev)))
        return nullptr;
    if (dev < 0 || dev >= kMaxDevices) {
        fmvd::report_error("fmvd: fmvd_b200_deconvolve_device_noalloc supports device ordinals below 64");
        return nullptr;
    }
    std::lock_guard<std::mutex> guard(g_setup_lock);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        if (!FMVD_CHECK(cudaGetSymbolAddress(&p, g_scratch)))
            return nullptr;
        g_scratch_addr[dev] = p;
    }
    return g_scratch_addr[dev];
}

} // namespace

extern "C" int fmvd_b200_deconvolve_device_noalloc(fmvd_b200_plan *plan, const void *d_views, size_t view_stride,
                                                   void *d_out, int nplanes, int iterations, float *d_estimate,
                                                   void *stream)
{
    if (!plan || !plan->eng || nplanes < 0) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_deconvolve_device_noalloc");
        return 1;
    }
    const fmvd::Engine *e = plan->eng;
    const size_t points = (size_t)e->dims.H * e->dims.W;
    const size_t pair_bytes = 2 * sizeof(float2) * points;  // complex work plane + estimate pair
    const size_t fit = (kScratchBytes - kStatusBytes) / pair_bytes;
    if (fit < 1) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "fmvd: fmvd_b200_deconvolve_device_noalloc: a %d x %d plane needs %zu bytes of work memory per "
                 "plane pair, more than its fixed %zu bytes; use fmvd_b200_deconvolve_device",
                 e->dims.H, e->dims.W, pair_bytes, kScratchBytes - kStatusBytes);
        fmvd::report_error(msg);
        return 1;
    }
    char *base = static_cast<char *>(scratch_address());
    if (!base)
        return 1;
    const cudaStream_t s = (cudaStream_t)stream;

    // The plan's spectra, weights and twiddles with the work memory swapped
    // for the shared array.
    fmvd::Engine run = *e;
    run.pairs_cap = (int)(fit < (size_t)e->pairs_cap ? fit : (size_t)e->pairs_cap);
    run.status = reinterpret_cast<int *>(base);
    run.C = reinterpret_cast<float2 *>(base + kStatusBytes);
    run.est = run.C + (size_t)run.pairs_cap * points;
    run.lanes = 1;  // one set of work planes: the shared array

    if (!FMVD_CHECK(cudaMemsetAsync(run.status, 0, sizeof(int), s)))
        return 1;
    if (!fmvd::engine_run(&run, d_views, view_stride, d_out, nplanes, iterations, d_estimate, s))
        return 1;
    // The status word is reused by the next call, so it is read before
    // returning: the call waits for its work on the stream to finish.
    int status = 0;
    if (!FMVD_CHECK(cudaStreamSynchronize(s)) ||
        !FMVD_CHECK(cudaMemcpy(&status, run.status, sizeof(int), cudaMemcpyDeviceToHost)))
        return 1;
    if (status) {
        fmvd::report_error("fmvd: a bulk copy into shared memory did not complete in time");
        return 1;
    }
    return 0;
}
