// Internal declarations shared by the host-side translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdio.h>

#include "fmvd_types.h"
#include "rl_kernels.h"

namespace fmvd {

// ---- error convention (fmvd_cuda_utils.cpp)
void report_error(const char *message);
bool check_cuda(unsigned int code, const char *file, int line);
void set_error_handler(void (*handler)(void *, const char *), void *param);
int idiv_up(int a, int b);
void get_last_cuda_error(const char *msg, const char *file, int line);
int num_devices();
void device_name(int dev, char *name);
void set_device(int dev);

#define FMVD_CHECK(call) ::fmvd::check_cuda((unsigned int)(call), __FILE__, __LINE__)

// ---- RL engine: kernel spectra, weights and work buffers of one plan
struct Engine {
    RlDims dims;
    int kH, kW;
    int pairs_cap;          // plane pairs per batch
    int device;
    size_t spec_elems;      // complex values per kernel spectrum (launch layout)
    float2 *spec;           // V x 2 spectra: [v][0] kernel 1, [v][1] kernel 2
    float *weights;         // V x dataH x dataW normalised weights
    float2 *C;              // pairs_cap x H x W
    float2 *est;            // pairs_cap x H x W
    float2 *twH, *twW;      // exp(-2 pi i n / N), line engine (lengths above 1024)
    float2 *wtwH, *wtwW;    // warp engine twiddle tables
    int *status;            // device flag: a bulk-copy wait timed out
    // Second lane: alternate batches run on a side stream with their own
    // work planes, so one batch's passes fill the idle SMs of the other's
    // last waves (lanes = 1: a single lane, no side stream).
    int lanes;
    float2 *laneC[3], *laneEst[3];   // lanes 1.. : pairs_cap x H x W each
    cudaStream_t side[3];
    cudaEvent_t ev_fork, ev_join[3];
};

// Lanes of a device plan (batches in flight on separate streams).
#ifndef FMVD_ENGINE_LANES
#define FMVD_ENGINE_LANES 2
#endif
constexpr int kMaxLanes = 4;

// Build an engine.  h_Kernel is normalised in place (reference semantics).
// pairs_cap <= 0 selects the default batch size.  Returns null after
// reporting an error.
// col_warps: column-pass warps per block (2, 4 or 8; 0 = widest that fits).
// lanes: FMVD_ENGINE_LANES for device plans (engine_run deals batches
// round-robin over that many work buffer sets and streams), 1 where the
// caller pipelines batches itself.  pairs_cap <= 0: the L2-sized default,
// split over the lanes.
Engine *engine_create(int bits, int dataH, int dataW, const float *const *h_Weights, float **h_Kernel, int kH,
                      int kW, int psf_type, int nViews, int pairs_cap, int col_warps = 0,
                      int lanes = FMVD_ENGINE_LANES);
void engine_destroy(Engine *e);
int default_pairs_cap(int H, int W, int lanes = 1);

// Deconvolve nplanes planes resident on the device.  View v, plane z of the
// input is at data + (v * view_stride + z * plane) samples; plane z of the
// output at out + z * plane.  est_out (optional) receives nplanes float
// planes of H x W.  Planes are processed in batches of 2 * pairs_cap.
// init (optional): nplanes float planes of H x W to start from instead of the
// reference's constant 10 * nViews; running k iterations from the estimate
// that j iterations returned gives the result of j + k iterations.
bool engine_run(Engine *e, const void *data, size_t view_stride, void *out, int nplanes, int iterations,
                float *est_out, cudaStream_t s, const float *init = nullptr);

// Reports (and clears) a timed-out bulk-copy wait flagged by the kernels;
// false if one was flagged.  Synchronises with the device.
bool engine_check_status(Engine *e);

// Launch sequence of one batch (at most 2 * pairs_cap planes).
void engine_batch(Engine *e, const void *data, size_t view_stride, void *out, int nplanes, int iterations,
                  cudaStream_t s, const float *init = nullptr);

// ---- plans and streaming (deconvolve.cpp)
void *pinned_malloc(size_t size);
void pinned_free(void *p);
// Whether p is still a pinned host allocation of the process's CUDA context.
// Pinned buffers kept for reuse are checked with it: cudaDeviceReset releases
// them behind the cache's back.
bool pinned_still_valid(const void *p);
fmvd_plan_cuda_16 *initialize_16(int dataH, int dataW, const float *const *w, float **k, int kH, int kW, int type,
                                 int V, int nstreams, datasource_16_t src, datasink_16_t sink, int pairs_cap);
fmvd_plan_cuda_8 *initialize_8(int dataH, int dataW, const float *const *w, float **k, int kH, int kW, int type,
                               int V, int nstreams, datasource_8_t src, datasink_8_t sink, int pairs_cap);
void deconvolve_planes_16(const fmvd_plan_cuda_16 *p, int iterations);
void deconvolve_planes_8(const fmvd_plan_cuda_8 *p, int iterations);
void destroy_16(fmvd_plan_cuda_16 *p);
void destroy_8(fmvd_plan_cuda_8 *p);
void deconvolve_files_16(FILE **f, FILE *r, int dW, int dH, int dD, float **w, float **k, int kH, int kW, int type,
                         int V, int it);
void deconvolve_files_8(FILE **f, FILE *r, int dW, int dH, int dD, float **w, float **k, int kH, int kW, int type,
                        int V, int it);
Engine *plan_engine_16(const fmvd_plan_cuda_16 *p);
Engine *plan_engine_8(const fmvd_plan_cuda_8 *p);

// ---- convergence statistics and warm-start padding (stats.cu)
bool plane_stats(const float *a, const float *b, int nplanes, int H, int W, int rows, int cols, double *out,
                 cudaStream_t s);
bool pad_estimate(const float *in, float *out, int nplanes, const RlDims &d, float floor_value, cudaStream_t s);

// ---- resampler (transform.cu)
void transform_file(int bits, const void *const *h_planes, int w, int h, int d, int tw, int th, int td,
                    const float *h_inverse, const char *outfile, int masks, int border, float zspacing,
                    const char *maskfile);

} // namespace fmvd

// Device-resident plan of the fmvd_b200_* entry points.
struct fmvd_b200_plan {
    fmvd::Engine *eng;
};
