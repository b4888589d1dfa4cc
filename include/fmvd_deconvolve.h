/* Plane-wise multi-view Richardson-Lucy deconvolution, C ABI.
 *
 * Drop-in replacement for the reference's public deconvolution API; each
 * entry point keeps the reference's name, arguments, ownership and error
 * behaviour (errors go to the handler installed with setErrorHandler):
 *
 *   fmvd_malloc / fmvd_free                    fmvd_deconvolve.h:11-15, fmvd_deconvolve.cpp:206-218
 *   fmvd_initialize_cuda_16 / _8               fmvd_deconvolve.impl.h:41-50, fmvd_deconvolve.impl.cpp:130-203
 *   fmvd_deconvolve_planes_cuda_16 / _8        fmvd_deconvolve.impl.h:53-54, fmvd_deconvolve.impl.cpp:205-300
 *   fmvd_destroy_cuda_16 / _8                  fmvd_deconvolve.impl.h:56-57, fmvd_deconvolve.impl.cpp:302-336
 *   fmvd_deconvolve_files_cuda_16 / _8         fmvd_deconvolve.impl.h:59-66, fmvd_deconvolve_hdd.impl.cpp:36-76
 *
 * The reference declares these with C++ linkage; this library exports them
 * both with C linkage (this header) and with the reference's C++ linkage, so
 * C++ code built against the reference headers links unchanged.
 *
 * Semantics kept from the reference:
 *  - h_Kernel is normalised in place (sum 1) after kernel 2 has been derived
 *    from the unnormalised kernels;
 *  - the FFT plane is snapTransformSize(data + kernel - 1) per axis;
 *  - views update the estimate in order; the estimate starts at 10 * nViews;
 *  - output is cropped, clipped at 2^bits - 1 and truncated;
 *  - fmvd_deconvolve_planes_cuda_* calls the datasource until it returns 0
 *    and the datasink once per plane in z order; a source with fewer planes
 *    than nstreams still yields nstreams sink calls (the reference processes
 *    its unfilled slots; here they are planes of zero data).
 * Differences: the library reads ahead by a whole batch of planes before the
 * first sink call (the reference reads ahead nstreams planes), and planes
 * wider or taller than 4096 after padding are rejected through the error
 * handler.
 */
#ifndef FMVD_DECONVOLVE_H
#define FMVD_DECONVOLVE_H

#include <stdio.h>
#include "fmvd_types.h"

#ifdef __cplusplus
extern "C" {
#endif

void *fmvd_malloc(size_t size);
void fmvd_free(void *p);

struct fmvd_plan_cuda_16 *fmvd_initialize_cuda_16(int dataH, int dataW, float const *const *h_Weights,
                                                  float **h_Kernel, int kernelH, int kernelW,
                                                  fmvd_psf_type iteration_type, int nViews, int nstreams,
                                                  datasource_16_t get_next_plane, datasink_16_t return_next_plane);
void fmvd_deconvolve_planes_cuda_16(const struct fmvd_plan_cuda_16 *plan, int iterations);
void fmvd_destroy_cuda_16(struct fmvd_plan_cuda_16 *plan);
void fmvd_deconvolve_files_cuda_16(FILE **dataFiles, FILE *resultFile, int dataW, int dataH, int dataD,
                                   float **h_Weights, float **h_Kernel, int kernelH, int kernelW,
                                   fmvd_psf_type iteration_type, int nViews, int iterations);

struct fmvd_plan_cuda_8 *fmvd_initialize_cuda_8(int dataH, int dataW, float const *const *h_Weights,
                                                float **h_Kernel, int kernelH, int kernelW,
                                                fmvd_psf_type iteration_type, int nViews, int nstreams,
                                                datasource_8_t get_next_plane, datasink_8_t return_next_plane);
void fmvd_deconvolve_planes_cuda_8(const struct fmvd_plan_cuda_8 *plan, int iterations);
void fmvd_destroy_cuda_8(struct fmvd_plan_cuda_8 *plan);
void fmvd_deconvolve_files_cuda_8(FILE **dataFiles, FILE *resultFile, int dataW, int dataH, int dataD,
                                  float **h_Weights, float **h_Kernel, int kernelH, int kernelW,
                                  fmvd_psf_type iteration_type, int nViews, int iterations);

#ifdef __cplusplus
}
#endif

#endif /* FMVD_DECONVOLVE_H */
