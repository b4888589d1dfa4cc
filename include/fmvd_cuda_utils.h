/* Error handling and device selection, C ABI.
 *
 * Replaces fmvd_cuda_utils.h:4-25 of the reference (same names and
 * behaviour; the reference declares them with C++ linkage and this library
 * exports both linkages):
 *   setErrorHandler     install the callback invoked with a message on any
 *                       CUDA or argument error (default: print and exit)
 *   iDivUp              ceil(a / b) for positive ints
 *   __getLastCudaError  report cudaGetLastError() if set
 *   __gpuAssert         report a failing CUDA status code
 *   getNumCUDADevices / getCudaDeviceName (name: 256 bytes) / setCudaDevice
 */
#ifndef FMVD_CUDA_UTILS_H
#define FMVD_CUDA_UTILS_H

#ifdef __cplusplus
extern "C" {
#endif

void setErrorHandler(void (*handler)(void *, const char *), void *param);
int iDivUp(int a, int b);
void __getLastCudaError(const char *errorMessage, const char *file, const int line);
void __gpuAssert(unsigned int code, const char *file, int line);
int getNumCUDADevices(void);
void getCudaDeviceName(int dev, char *name);
void setCudaDevice(int dev);

#ifdef __cplusplus
}
#endif

#define getLastCudaError(msg) __getLastCudaError(msg, __FILE__, __LINE__)
#define checkCudaErrors(ans) \
    { __gpuAssert((ans), __FILE__, __LINE__); }

#endif /* FMVD_CUDA_UTILS_H */
