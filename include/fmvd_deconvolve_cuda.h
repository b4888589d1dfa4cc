/* Element-wise device launchers of the reference's public CUDA header
 * (fmvd_deconvolve_cuda.cuh:20-90, fmvd_deconvolve_cuda.impl.cuh:6-37), C ABI.
 *
 * The deconvolution itself does not use them (its passes are fused); they
 * are exported with the reference's names, arguments and semantics so that
 * code calling them keeps working.  All pointers are device memory; every
 * launcher is asynchronous on 'stream'.
 *
 *   padKernel                 zero-filled fftH x fftW destination expected;
 *                             writes the kernel with centre (kH/2, kW/2) at (0, 0)
 *   padWeights                clamp-to-border pad, accumulates into the sums
 *   normalizeWeights          w /= sum where sum > 0
 *   padDataClampToBorder32    clamp-to-border pad (borders kH/2 rows, kW/2 columns)
 *   unpadData32               crop
 *   modulateAndNormalize      dst = src * dst / (fftW * fftH), fftH * (fftW/2 + padding) values
 *   multiply32                dest += weights * (a * b - dest)
 *   padDataClampToBorderAndInitialize_N
 *                             pad samples, estimate += 10 (the reference's 9th and
 *                             10th parameters arrive as (kernelH, kernelW) from
 *                             its caller but are named (kernelW, kernelH): the row
 *                             border is parameter 10 / 2, the column border
 *                             parameter 9 / 2)
 *   unpadData_N               crop, clip at the sample maximum, truncate
 *   divide_N                  dest = a / b where b > 1
 */
#ifndef FMVD_DECONVOLVE_CUDA_H
#define FMVD_DECONVOLVE_CUDA_H

#include <cuda_runtime.h>
#include "fmvd_types.h"

#ifdef __cplusplus
extern "C" {
#endif

void padKernel(float *d_PaddedKernel, float *d_Kernel, int fftH, int fftW, int kernelH, int kernelW,
               cudaStream_t stream);
void padWeights(float *d_PaddedWeights, float *d_PaddedWeightSums, float *d_Weights, int fftH, int fftW, int dataH,
                int dataW, int kernelH, int kernelW, cudaStream_t stream);
void normalizeWeights(float *d_PaddedWeights, float *d_PaddedWeightSums, int fftH, int fftW, cudaStream_t stream);
void padDataClampToBorder32(float *d_PaddedData, float *d_Data, int fftH, int fftW, int dataH, int dataW, int kernelH,
                            int kernelW, cudaStream_t stream);
void unpadData32(float *d_Dst, float *d_Src, int fftH, int fftW, int dataH, int dataW, cudaStream_t stream);
void modulateAndNormalize(fComplex *d_Dst, fComplex *d_Src, int fftH, int fftW, int padding, cudaStream_t stream);
void multiply32(float *d_a, float *d_b, float *d_weights, float *d_dest, int fftH, int fftW, cudaStream_t stream);

void padDataClampToBorderAndInitialize_16(float *d_estimate, unsigned short *d_PaddedData, unsigned short *d_Data,
                                          float *d_Weights, int fftH, int fftW, int dataH, int dataW, int kernelH,
                                          int kernelW, cudaStream_t stream);
void unpadData_16(unsigned short *d_Data, float *d_PaddedData, int fftH, int fftW, int dataH, int dataW,
                  cudaStream_t stream);
void divide_16(unsigned short *d_a, float *d_b, float *d_dest, int fftH, int fftW, cudaStream_t stream);

void padDataClampToBorderAndInitialize_8(float *d_estimate, unsigned char *d_PaddedData, unsigned char *d_Data,
                                         float *d_Weights, int fftH, int fftW, int dataH, int dataW, int kernelH,
                                         int kernelW, cudaStream_t stream);
void unpadData_8(unsigned char *d_Data, float *d_PaddedData, int fftH, int fftW, int dataH, int dataW,
                 cudaStream_t stream);
void divide_8(unsigned char *d_a, float *d_b, float *d_dest, int fftH, int fftW, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* FMVD_DECONVOLVE_CUDA_H */
