// Device-side resampler entry points (transform.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <mutex>

namespace fmvd {

// Row pitch (samples) of the device source volume: rows padded to 16 bytes
// so that the TMA tensor map's strides are legal.
size_t source_pitch(int bits, int w);

// Resample target planes [z0, z0 + nz) of a tw x th x td frame from a source
// volume in device memory (d planes, h rows, 'pitch' samples per row).
// d_out receives nz planes of samples (or null), d_outf nz float planes in
// sample units (or null).  d_status is set to 1 if a brick load timed out.
bool resample_device(int bits, const void *d_src, size_t pitch, int w, int h, int d, int tw, int th, int z0, int nz,
                     const float *h_inverse, void *d_out, float *d_outf, int *d_status, cudaStream_t s);
void resample_direct(int bits, const void *d_src, size_t pitch, int w, int h, int d, int tw, int th, int z0, int nz,
                     const float *h_inverse, void *d_out, float *d_outf, cudaStream_t s);
// Pinned staging buffers (index 0..3) kept for the life of the process,
// grown on demand; hold staging_lock() while using them.
std::unique_lock<std::mutex> staging_lock();
void *staging_buffer(int i, size_t bytes);
// memcpy of a large block split over a few host threads.
void host_copy(void *dst, const void *src, size_t bytes);
// Upload of d source planes (host pointers into any host memory, w samples
// per row, h rows) into the pitched device volume d_src through two pinned
// staging buffers used in turn; returns once the copies have landed.
bool upload_planes(const void *const *h_planes, int w, int h, int d, size_t es, size_t pitch, void *d_src,
                   cudaStream_t s);
// Transformed weight mask of target plane z (tw x th floats).
bool mask_device(float *d_out, int z, int w, int h, int d, float zspacing, int tw, int th, float border,
                 const float *h_inverse, cudaStream_t s);

} // namespace fmvd
