/* Types shared by the public headers of the B200 multi-view reconstruction
 * library (drop-in for bene51/gpu_deconvolution).
 *
 * Names and meanings follow the reference headers:
 *   fmvd_psf_type           fmvd_deconvolve.h:9
 *   datasource_N_t / datasink_N_t, struct fmvd_plan_cuda_N
 *                           fmvd_deconvolve.impl.h:5-64
 *   fComplex                fmvd_deconvolve_cuda.cuh:10-17
 * The plan structs keep the reference's leading geometry fields (dataH,
 * dataW, fftH, fftW, kernelH, kernelW, nViews, nStreams) in the same order;
 * the device buffers behind them are private to the library.
 */
#ifndef FMVD_TYPES_H
#define FMVD_TYPES_H

#include <stddef.h>

#ifdef __CUDACC__
#include <vector_types.h>
typedef float2 fComplex;
#else
typedef struct {
    float x;
    float y;
} fComplex;
#endif

typedef enum fmvd_psf_type { independent, efficient_bayesian, optimization_1, optimization_2 } fmvd_psf_type;

/* Fills buffer[v] + offset (one plane, dataH * dataW samples, per view v);
 * returns 0 once no more planes are available. */
typedef int (*datasource_16_t)(unsigned short **buffer, int offset);
typedef int (*datasource_8_t)(unsigned char **buffer, int offset);
/* Receives one deconvolved plane (dataH * dataW samples), in z order; the
 * pointer is valid for the duration of the call. */
typedef void (*datasink_16_t)(unsigned short *buffer);
typedef void (*datasink_8_t)(unsigned char *buffer);

struct fmvd_plan_cuda_16 {
    int dataH, dataW;
    int fftH, fftW;
    int kernelH, kernelW;
    int nViews;
    int nStreams;
    datasource_16_t get_next_plane;
    datasink_16_t return_next_plane;
    void *engine; /* private */
};

struct fmvd_plan_cuda_8 {
    int dataH, dataW;
    int fftH, fftW;
    int kernelH, kernelW;
    int nViews;
    int nStreams;
    datasource_8_t get_next_plane;
    datasink_8_t return_next_plane;
    void *engine; /* private */
};

#ifndef __cplusplus
typedef struct fmvd_plan_cuda_16 fmvd_plan_cuda_16;
typedef struct fmvd_plan_cuda_8 fmvd_plan_cuda_8;
#endif

#endif /* FMVD_TYPES_H */
