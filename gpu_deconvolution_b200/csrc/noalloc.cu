// fmvd_b200_deconvolve_device_noalloc: the device-resident deconvolution of
// a plan with its work memory taken from a fixed array of this library, so the
// call itself allocates nothing.
//
// Why: some callers cannot call cudaMalloc at the point where they
// deconvolve.  A host framework that owns the device's free memory through
// its own pool, a real-time acquisition loop that must not take the
// allocator's device-wide synchronisation, or a plugin running inside another
// application's CUDA context may only hand this library buffers it already
// holds.  fmvd_b200_deconvolve_device itself allocates nothing either, but it
// runs in work planes the plan allocated at creation, sized for the plan's
// batch and lanes; this entry point runs in one array of this library that
// the CUDA runtime reserves when it loads the library's module on a device,
// so the call needs no memory beyond the plan's spectra and weights and the
// caller's inputs and outputs.  The plan still holds its own work planes
// (created with pairs_per_batch = 1 they are the smallest the plan allows);
// this entry point does not use them.  Nothing here calls cudaMalloc,
// cudaFree or any routine that allocates.
//
// Limit: the array is kScratchBytes (64 MiB).  Its first 256 bytes hold the
// wait-status word; the rest holds the work planes of as many plane pairs as
// fit, at most the plan's own batch size.  A plan whose padded plane does not
// fit one pair (more than about 4.19 M complex points, e.g. 2048 x 2048) is
// rejected with an error.
//
// Device: the call must be made with the plan's device current (the array is
// per device); another current device is rejected.  The array's device
// address is looked up on every call (cudaGetSymbolAddress allocates
// nothing).  The first call on a device may make the runtime load the
// library's module there, so make that first call before any stream capture.
//
// Sharing: every call on a device uses the same array, and the array keeps
// the last call's contents.  The status word is cleared at the start of each
// call; the work planes are written before they are read.  Calls that
// overlap in time on one device (from two host threads, or queued on two
// streams) race on the array and corrupt each other's results: serialise them.
// The call returns only when its work on the stream has finished, on success
// and on failure, so consecutive calls from one thread never overlap.
#include "fmvd_b200.h"
#include "fmvd_internal.h"

#include <stdio.h>

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr size_t kStatusBytes = 256;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch on the current device (an error is reported
// and null returned if the lookup fails).
void *scratch_address()
{
    void *p = nullptr;
    if (!FMVD_CHECK(cudaGetSymbolAddress(&p, g_scratch)))
        return nullptr;
    return p;
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
    int dev = -1;
    if (!FMVD_CHECK(cudaGetDevice(&dev)))
        return 1;
    if (dev != e->device) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "fmvd: fmvd_b200_deconvolve_device_noalloc: the plan lives on device %d but device %d is current",
                 e->device, dev);
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
    if (!fmvd::engine_run(&run, d_views, view_stride, d_out, nplanes, iterations, d_estimate, s)) {
        // kernels queued before the failure still use the array: let them
        // finish so that the array is idle when this call returns
        cudaStreamSynchronize(s);
        return 1;
    }
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
