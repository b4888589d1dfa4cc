// Error reporting and device utilities of the public ABI
// (replaces fmvd_cuda_utils.cpp:12-85 of the reference; same names, argument
// meaning and error behaviour: a failing CUDA call reports
// "Cuda error <code>: <text> in <file> (line <n>)" on stderr and invokes the
// installed handler, whose default terminates the process).
#include "fmvd_internal.h"

#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

namespace {

void default_handler(void *, const char *)
{
    printf("exiting... \n");
    exit(EXIT_FAILURE);
}

void (*g_handler)(void *, const char *) = default_handler;
void *g_handler_param = NULL;

} // namespace

namespace fmvd {

void report_error(const char *message)
{
    fprintf(stderr, "%s\n", message);
    g_handler(g_handler_param, message);
}

bool check_cuda(unsigned int code, const char *file, int line)
{
    if (code == cudaSuccess)
        return true;
    char message[256];
    snprintf(message, sizeof(message), "Cuda error %d: %s in %s (line %i)", (int)code,
             cudaGetErrorString((cudaError_t)code), file, line);
    report_error(message);
    return false;
}

} // namespace fmvd

namespace fmvd {

void set_error_handler(void (*handler)(void *, const char *), void *param)
{
    g_handler_param = param;
    g_handler = handler ? handler : default_handler;
}

int idiv_up(int a, int b) { return (a % b != 0) ? (a / b + 1) : (a / b); }

void get_last_cuda_error(const char *, const char *file, int line) { check_cuda(cudaGetLastError(), file, line); }

int num_devices()
{
    int count = 0;
    check_cuda(cudaGetDeviceCount(&count), __FILE__, __LINE__);
    return count;
}

void device_name(int dev, char *name)
{
    cudaDeviceProp prop;
    if (check_cuda(cudaGetDeviceProperties(&prop, dev), __FILE__, __LINE__))
        memcpy(name, prop.name, 256);
}

void set_device(int dev) { check_cuda(cudaSetDevice(dev), __FILE__, __LINE__); }

} // namespace fmvd
