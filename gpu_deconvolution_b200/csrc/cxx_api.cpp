// C++-linkage exports with the reference's exact signatures, so that code
// compiled against the reference headers (where these functions have C++
// linkage: fmvd_deconvolve.impl.h:41-66, fmvd_transform.h:4-24,
// fmvd_cuda_utils.h:4-25, fmvd_deconvolve.h:11-15) links against this
// library without change.  This file deliberately does not include the
// library's own C-linkage headers.
#include <stdio.h>

#include "fmvd_types.h"
#include "fmvd_internal.h"

void setErrorHandler(void (*handler)(void *, const char *), void *param) { fmvd::set_error_handler(handler, param); }
int iDivUp(int a, int b) { return fmvd::idiv_up(a, b); }
void __getLastCudaError(const char *m, const char *file, const int line) { fmvd::get_last_cuda_error(m, file, line); }
void __gpuAssert(unsigned int code, const char *file, int line) { fmvd::check_cuda(code, file, line); }
int getNumCUDADevices() { return fmvd::num_devices(); }
void getCudaDeviceName(int dev, char *name) { fmvd::device_name(dev, name); }
void setCudaDevice(int dev) { fmvd::set_device(dev); }

void *fmvd_malloc(size_t size) { return fmvd::pinned_malloc(size); }
void fmvd_free(void *p) { fmvd::pinned_free(p); }

fmvd_plan_cuda_16 *fmvd_initialize_cuda_16(int dataH, int dataW, float const *const *h_Weights, float **h_Kernel,
                                           int kernelH, int kernelW, fmvd_psf_type t, int nViews, int nstreams,
                                           datasource_16_t src, datasink_16_t sink)
{
    return fmvd::initialize_16(dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, t, nViews, nstreams, src, sink, 0);
}
void fmvd_deconvolve_planes_cuda_16(const fmvd_plan_cuda_16 *plan, int iterations)
{
    fmvd::deconvolve_planes_16(plan, iterations);
}
void fmvd_destroy_cuda_16(fmvd_plan_cuda_16 *plan) { fmvd::destroy_16(plan); }
void fmvd_deconvolve_files_cuda_16(FILE **dataFiles, FILE *resultFile, int dataW, int dataH, int dataD,
                                   float **h_Weights, float **h_Kernel, int kernelH, int kernelW, fmvd_psf_type t,
                                   int nViews, int iterations)
{
    fmvd::deconvolve_files_16(dataFiles, resultFile, dataW, dataH, dataD, h_Weights, h_Kernel, kernelH, kernelW, t,
                              nViews, iterations);
}

fmvd_plan_cuda_8 *fmvd_initialize_cuda_8(int dataH, int dataW, float const *const *h_Weights, float **h_Kernel,
                                         int kernelH, int kernelW, fmvd_psf_type t, int nViews, int nstreams,
                                         datasource_8_t src, datasink_8_t sink)
{
    return fmvd::initialize_8(dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, t, nViews, nstreams, src, sink, 0);
}
void fmvd_deconvolve_planes_cuda_8(const fmvd_plan_cuda_8 *plan, int iterations)
{
    fmvd::deconvolve_planes_8(plan, iterations);
}
void fmvd_destroy_cuda_8(fmvd_plan_cuda_8 *plan) { fmvd::destroy_8(plan); }
void fmvd_deconvolve_files_cuda_8(FILE **dataFiles, FILE *resultFile, int dataW, int dataH, int dataD,
                                  float **h_Weights, float **h_Kernel, int kernelH, int kernelW, fmvd_psf_type t,
                                  int nViews, int iterations)
{
    fmvd::deconvolve_files_8(dataFiles, resultFile, dataW, dataH, dataD, h_Weights, h_Kernel, kernelH, kernelW, t,
                             nViews, iterations);
}

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
