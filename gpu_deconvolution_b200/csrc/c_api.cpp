// C-linkage exports: the reference API names (include/fmvd_deconvolve.h,
// fmvd_transform.h, fmvd_cuda_utils.h) and the library extensions
// (include/fmvd_b200.h).
#include "fmvd_b200.h"
#include "fmvd_cuda_utils.h"
#include "fmvd_deconvolve.h"
#include "fmvd_internal.h"
#include "fmvd_transform.h"
#include "transform_kernels.h"

#include <string.h>
#include <vector>

extern "C" {

// ---- fmvd_cuda_utils.h
void setErrorHandler(void (*handler)(void *, const char *), void *param) { fmvd::set_error_handler(handler, param); }
int iDivUp(int a, int b) { return fmvd::idiv_up(a, b); }
void __getLastCudaError(const char *m, const char *file, const int line) { fmvd::get_last_cuda_error(m, file, line); }
void __gpuAssert(unsigned int code, const char *file, int line) { fmvd::check_cuda(code, file, line); }
int getNumCUDADevices(void) { return fmvd::num_devices(); }
void getCudaDeviceName(int dev, char *name) { fmvd::device_name(dev, name); }
void setCudaDevice(int dev) { fmvd::set_device(dev); }

// ---- fmvd_deconvolve.h
void *fmvd_malloc(size_t size) { return fmvd::pinned_malloc(size); }
void fmvd_free(void *p) { fmvd::pinned_free(p); }

struct fmvd_plan_cuda_16 *fmvd_initialize_cuda_16(int dataH, int dataW, float const *const *h_Weights,
                                                  float **h_Kernel, int kernelH, int kernelW,
                                                  fmvd_psf_type iteration_type, int nViews, int nstreams,
                                                  datasource_16_t src, datasink_16_t sink)
{
    return fmvd::initialize_16(dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, iteration_type, nViews, nstreams,
                               src, sink, 0);
}
void fmvd_deconvolve_planes_cuda_16(const struct fmvd_plan_cuda_16 *plan, int iterations)
{
    fmvd::deconvolve_planes_16(plan, iterations);
}
void fmvd_destroy_cuda_16(struct fmvd_plan_cuda_16 *plan) { fmvd::destroy_16(plan); }
void fmvd_deconvolve_files_cuda_16(FILE **dataFiles, FILE *resultFile, int dataW, int dataH, int dataD,
                                   float **h_Weights, float **h_Kernel, int kernelH, int kernelW,
                                   fmvd_psf_type iteration_type, int nViews, int iterations)
{
    fmvd::deconvolve_files_16(dataFiles, resultFile, dataW, dataH, dataD, h_Weights, h_Kernel, kernelH, kernelW,
                              iteration_type, nViews, iterations);
}

struct fmvd_plan_cuda_8 *fmvd_initialize_cuda_8(int dataH, int dataW, float const *const *h_Weights, float **h_Kernel,
                                                int kernelH, int kernelW, fmvd_psf_type iteration_type, int nViews,
                                                int nstreams, datasource_8_t src, datasink_8_t sink)
{
    return fmvd::initialize_8(dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, iteration_type, nViews, nstreams,
                              src, sink, 0);
}
void fmvd_deconvolve_planes_cuda_8(const struct fmvd_plan_cuda_8 *plan, int iterations)
{
    fmvd::deconvolve_planes_8(plan, iterations);
}
void fmvd_destroy_cuda_8(struct fmvd_plan_cuda_8 *plan) { fmvd::destroy_8(plan); }
void fmvd_deconvolve_files_cuda_8(FILE **dataFiles, FILE *resultFile, int dataW, int dataH, int dataD,
                                  float **h_Weights, float **h_Kernel, int kernelH, int kernelW,
                                  fmvd_psf_type iteration_type, int nViews, int iterations)
{
    fmvd::deconvolve_files_8(dataFiles, resultFile, dataW, dataH, dataD, h_Weights, h_Kernel, kernelH, kernelW,
                             iteration_type, nViews, iterations);
}

// ---- fmvd_transform.h
void transform_cuda_8(unsigned char **h_data, int w, int h, int d, int tw, int th, int td, float *h_inverse,
                      const char *outfile, int createTransformedMasks, int border, float zspacing,
                      const char *maskfile)
{
    fmvd::transform_file(8, (const void *const *)h_data, w, h, d, tw, th, td, h_inverse, outfile,
                         createTransformedMasks, border, zspacing, maskfile);
}

void transform_cuda_16(unsigned short **h_data, int w, int h, int d, int tw, int th, int td, float *h_inverse,
                       const char *outfile, int createTransformedMasks, int border, float zspacing,
                       const char *maskfile)
{
    fmvd::transform_file(16, (const void *const *)h_data, w, h, d, tw, th, td, h_inverse, outfile,
                         createTransformedMasks, border, zspacing, maskfile);
}

// ---- fmvd_b200.h
fmvd_b200_plan *fmvd_b200_plan_create(int bits, int dataH, int dataW, const float *const *h_Weights, float **h_Kernel,
                                      int kernelH, int kernelW, fmvd_psf_type iteration_type, int nViews,
                                      int pairs_per_batch)
{
    fmvd::Engine *e = fmvd::engine_create(bits, dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, iteration_type,
                                          nViews, pairs_per_batch);
    if (!e)
        return nullptr;
    return new fmvd_b200_plan{e};
}

fmvd_b200_plan *fmvd_b200_plan_create_tuned(int bits, int dataH, int dataW, const float *const *h_Weights,
                                            float **h_Kernel, int kernelH, int kernelW, fmvd_psf_type iteration_type,
                                            int nViews, int pairs_per_batch, int col_warps)
{
    fmvd::Engine *e = fmvd::engine_create(bits, dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, iteration_type,
                                          nViews, pairs_per_batch, col_warps);
    if (!e)
        return nullptr;
    return new fmvd_b200_plan{e};
}

fmvd_b200_plan *fmvd_b200_plan_create_scheduled(int bits, int dataH, int dataW, const float *const *h_Weights,
                                                float **h_Kernel, int kernelH, int kernelW,
                                                fmvd_psf_type iteration_type, int nViews, int pairs_per_batch,
                                                int col_warps, int radix_step)
{
    if (radix_step < 0 || radix_step > 2) {
        fmvd::report_error("fmvd: radix_step must be 0, 1 or 2");
        return nullptr;
    }
    fmvd::Engine *e = fmvd::engine_create(bits, dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, iteration_type,
                                          nViews, pairs_per_batch, col_warps);
    if (!e)
        return nullptr;
    e->dims.radix_step = radix_step == 2 ? fmvd::kRadixSums : fmvd::kRadixDft;
    return new fmvd_b200_plan{e};
}

int fmvd_b200_plan_radix_step(const fmvd_b200_plan *plan)
{
    return plan ? (plan->eng->dims.radix_step == fmvd::kRadixSums ? 2 : 1) : -1;
}

int fmvd_b200_plan_col_warps(const fmvd_b200_plan *plan) { return plan ? plan->eng->dims.col_warps : -1; }

int fmvd_b200_plan_query(const fmvd_b200_plan *plan, int *fftH, int *fftW, int *pairs)
{
    if (!plan)
        return 1;
    if (fftH)
        *fftH = plan->eng->dims.H;
    if (fftW)
        *fftW = plan->eng->dims.W;
    if (pairs)
        *pairs = plan->eng->pairs_cap;
    return 0;
}

int fmvd_b200_deconvolve_device(fmvd_b200_plan *plan, const void *d_views, size_t view_stride, void *d_out,
                                int nplanes, int iterations, float *d_estimate, void *stream)
{
    if (!plan || nplanes < 0) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_deconvolve_device");
        return 1;
    }
    return fmvd::engine_run(plan->eng, d_views, view_stride, d_out, nplanes, iterations, d_estimate,
                            (cudaStream_t)stream)
               ? 0
               : 1;
}

int fmvd_b200_deconvolve_device_from(fmvd_b200_plan *plan, const void *d_views, size_t view_stride, void *d_out,
                                     int nplanes, int iterations, const float *d_init, float *d_estimate,
                                     void *stream)
{
    if (!plan || nplanes < 0 || !d_init) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_deconvolve_device_from");
        return 1;
    }
    return fmvd::engine_run(plan->eng, d_views, view_stride, d_out, nplanes, iterations, d_estimate,
                            (cudaStream_t)stream, d_init)
               ? 0
               : 1;
}

int fmvd_b200_pad_estimate(const fmvd_b200_plan *plan, const float *d_in, float *d_out, int nplanes,
                           float floor_value, void *stream)
{
    if (!plan || nplanes < 0 || (nplanes > 0 && (!d_in || !d_out))) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_pad_estimate");
        return 1;
    }
    return fmvd::pad_estimate(d_in, d_out, nplanes, plan->eng->dims, floor_value, (cudaStream_t)stream) ? 0 : 1;
}

int fmvd_b200_plane_stats(const float *d_a, const float *d_b, int nplanes, int H, int W, int rows, int cols,
                          double *d_stats, void *stream)
{
    if (nplanes < 0 || H <= 0 || W <= 0 || rows < 0 || cols < 0 || rows > H || cols > W ||
        (nplanes > 0 && (!d_a || !d_stats))) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_plane_stats");
        return 1;
    }
    return fmvd::plane_stats(d_a, d_b, nplanes, H, W, rows, cols, d_stats, (cudaStream_t)stream) ? 0 : 1;
}

int fmvd_b200_plan_check(fmvd_b200_plan *plan)
{
    if (!plan)
        return 1;
    return fmvd::engine_check_status(plan->eng) ? 0 : 1;
}

void fmvd_b200_plan_destroy(fmvd_b200_plan *plan)
{
    if (!plan)
        return;
    cudaDeviceSynchronize();
    fmvd::engine_destroy(plan->eng);
    delete plan;
}

struct fmvd_plan_cuda_16 *fmvd_b200_initialize_cuda_16(int dataH, int dataW, float const *const *h_Weights,
                                                       float **h_Kernel, int kernelH, int kernelW,
                                                       fmvd_psf_type iteration_type, int nViews, int nstreams,
                                                       datasource_16_t src, datasink_16_t sink, int pairs)
{
    return fmvd::initialize_16(dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, iteration_type, nViews, nstreams,
                               src, sink, pairs);
}

struct fmvd_plan_cuda_8 *fmvd_b200_initialize_cuda_8(int dataH, int dataW, float const *const *h_Weights,
                                                     float **h_Kernel, int kernelH, int kernelW,
                                                     fmvd_psf_type iteration_type, int nViews, int nstreams,
                                                     datasource_8_t src, datasink_8_t sink, int pairs)
{
    return fmvd::initialize_8(dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, iteration_type, nViews, nstreams,
                              src, sink, pairs);
}

size_t fmvd_b200_source_pitch(int bits, int w) { return fmvd::source_pitch(bits, w); }

int fmvd_b200_transform_device(int bits, const void *d_src, size_t pitch, int w, int h, int d, int tw, int th, int z0,
                               int nz, const float *h_inverse, void *d_out, float *d_outf, void *stream)
{
    if ((bits != 8 && bits != 16) || pitch % fmvd::source_pitch(bits, 1) != 0 || pitch < (size_t)w) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_transform_device");
        return 1;
    }
    int *d_status = nullptr;
    if (!FMVD_CHECK(cudaMallocAsync(&d_status, sizeof(int), (cudaStream_t)stream)))
        return 1;
    FMVD_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), (cudaStream_t)stream));
    const bool ok = fmvd::resample_device(bits, d_src, pitch, w, h, d, tw, th, z0, nz, h_inverse, d_out, d_outf,
                                          d_status, (cudaStream_t)stream);
    FMVD_CHECK(cudaFreeAsync(d_status, (cudaStream_t)stream));
    return ok ? 0 : 1;
}

int fmvd_b200_mask_device(float *d_out, int z, int w, int h, int d, float zspacing, int tw, int th, float border,
                          const float *h_inverse, void *stream)
{
    return fmvd::mask_device(d_out, z, w, h, d, zspacing, tw, th, border, h_inverse, (cudaStream_t)stream) ? 0 : 1;
}

int fmvd_b200_transform_host(int bits, const void *const *h_planes, int w, int h, int d, int tw, int th, int td,
                             const float *h_inverse, void *h_out)
{
    // upload through pinned staging, then resample in chunks of target
    // planes; each chunk's download to pinned staging and its copy into the
    // caller's buffer overlap the resampling of the next chunk (the staging
    // buffers are kept from call to call)
    auto lock = fmvd::staging_lock();
    const size_t es = bits == 16 ? 2 : 1;
    const size_t pitch = fmvd::source_pitch(bits, w);
    const size_t plane = (size_t)tw * th * es;
    int chunk = (int)(((size_t)16 << 20) / (plane ? plane : 1));
    chunk = chunk < 1 ? 1 : (chunk > td ? (td > 0 ? td : 1) : chunk);
    void *d_src = nullptr, *d_out = nullptr;
    void *stage[2] = {fmvd::staging_buffer(2, plane * chunk), fmvd::staging_buffer(3, plane * chunk)};
    int *d_status = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool ok = stage[0] && stage[1] && FMVD_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) &&
              FMVD_CHECK(cudaMalloc(&d_src, pitch * h * d * es)) &&
              FMVD_CHECK(cudaMalloc(&d_out, 2 * plane * chunk)) && FMVD_CHECK(cudaMalloc(&d_status, sizeof(int))) &&
              FMVD_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), s));
    for (int k = 0; k < 2 && ok; k++)
        ok = FMVD_CHECK(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
    ok = ok && fmvd::upload_planes(h_planes, w, h, d, es, pitch, d_src, s);
    int pending = -1, pending_z = 0, pending_n = 0;
    for (int z0 = 0, k = 0; ok && z0 < td; z0 += chunk, k ^= 1) {
        const int n = td - z0 < chunk ? td - z0 : chunk;
        char *dk = (char *)d_out + (size_t)k * plane * chunk;
        ok = fmvd::resample_device(bits, d_src, pitch, w, h, d, tw, th, z0, n, h_inverse, dk, nullptr, d_status, s) &&
             FMVD_CHECK(cudaMemcpyAsync(stage[k], dk, plane * n, cudaMemcpyDeviceToHost, s)) &&
             FMVD_CHECK(cudaEventRecord(ev[k], s));
        if (ok && pending >= 0) {
            ok = FMVD_CHECK(cudaEventSynchronize(ev[pending]));
            if (ok)
                fmvd::host_copy((char *)h_out + plane * pending_z, stage[pending], plane * pending_n);
        }
        pending = k;
        pending_z = z0;
        pending_n = n;
    }
    if (ok && pending >= 0) {
        ok = FMVD_CHECK(cudaEventSynchronize(ev[pending]));
        if (ok)
            fmvd::host_copy((char *)h_out + plane * pending_z, stage[pending], plane * pending_n);
    }
    int status = 0;
    if (s)
        cudaStreamSynchronize(s);
    if (ok)
        ok = FMVD_CHECK(cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (ok && status) {
        fmvd::report_error("fmvd: a resampler brick load did not complete in time");
        ok = false;
    }
    for (int k = 0; k < 2; k++)
        if (ev[k])
            cudaEventDestroy(ev[k]);
    cudaFree(d_src);
    cudaFree(d_out);
    cudaFree(d_status);
    if (s)
        cudaStreamDestroy(s);
    return ok ? 0 : 1;
}

unsigned long long fmvd_b200_launch_count(void) { return fmvd::rl_launch_count(); }

} // extern "C"
