/* Extensions of the B200 library beyond the reference API (no counterpart
 * in bene51/gpu_deconvolution).  All return 0 on success and a non-zero code
 * after reporting the error through the handler installed with
 * setErrorHandler.  Stream arguments are cudaStream_t values (0 = default
 * stream); device pointers are CUDA device memory of the current device.
 */
#ifndef FMVD_B200_H
#define FMVD_B200_H

#include <stddef.h>
#include "fmvd_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- device-resident deconvolution (no datasource / datasink) ---------- */
typedef struct fmvd_b200_plan fmvd_b200_plan;

/* Same preparation as fmvd_initialize_cuda_* (kernel 2 derivation, in-place
 * normalisation of h_Kernel, weight normalisation).  pairs_per_batch: plane
 * pairs deconvolved together (0 = automatic, sized for L2 residency). */
fmvd_b200_plan *fmvd_b200_plan_create(int bits, int dataH, int dataW, const float *const *h_Weights,
                                      float **h_Kernel, int kernelH, int kernelW, fmvd_psf_type iteration_type,
                                      int nViews, int pairs_per_batch);
int fmvd_b200_plan_query(const fmvd_b200_plan *plan, int *fftH, int *fftW, int *pairs_per_batch);
/* fmvd_b200_plan_create with the column-pass width as well: col_warps = 2, 4
 * or 8 warps (columns) per block for padded planes up to 1024 rows, 0 for
 * the widest the plane allows (the autotuner's two knobs are
 * pairs_per_batch and col_warps). */
fmvd_b200_plan *fmvd_b200_plan_create_tuned(int bits, int dataH, int dataW, const float *const *h_Weights,
                                            float **h_Kernel, int kernelH, int kernelW, fmvd_psf_type iteration_type,
                                            int nViews, int pairs_per_batch, int col_warps);
/* fmvd_b200_plan_create_tuned with the radix schedule of lines longer than
 * 1024 as well: radix_step = 1 runs the radix-R step of the R x 512 line
 * transforms as R-point DFTs per position, 2 as each sub-line group's
 * weighted sum over the R sub-lines (the same transform with a different
 * instruction mix), 0 the default (1).  The autotuner's third knob. */
fmvd_b200_plan *fmvd_b200_plan_create_scheduled(int bits, int dataH, int dataW, const float *const *h_Weights,
                                                float **h_Kernel, int kernelH, int kernelW,
                                                fmvd_psf_type iteration_type, int nViews, int pairs_per_batch,
                                                int col_warps, int radix_step);
/* The plan's radix schedule (1 or 2, as above). */
int fmvd_b200_plan_radix_step(const fmvd_b200_plan *plan);
/* Column-pass warps per block of the plan (0 for planes above 1024 rows,
 * whose column pass has a fixed two-column tile). */
int fmvd_b200_plan_col_warps(const fmvd_b200_plan *plan);
/* View v, plane z at d_views + (v * view_stride + z * dataH * dataW) samples;
 * output plane z at d_out + z * dataH * dataW.  d_estimate (optional)
 * receives nplanes float planes of fftH x fftW.  Asynchronous on stream. */
int fmvd_b200_deconvolve_device(fmvd_b200_plan *plan, const void *d_views, size_t view_stride, void *d_out,
                                int nplanes, int iterations, float *d_estimate, void *stream);
/* fmvd_b200_deconvolve_device starting from d_init (nplanes float planes of
 * fftH x fftW) instead of the constant 10 * nViews: iterations continue a
 * previous run exactly when d_init is the estimate that run returned, and
 * start from a warm-start estimate otherwise.  d_init may equal
 * d_estimate. */
int fmvd_b200_deconvolve_device_from(fmvd_b200_plan *plan, const void *d_views, size_t view_stride, void *d_out,
                                     int nplanes, int iterations, const float *d_init, float *d_estimate,
                                     void *stream);
/* Estimates on the data plane (nplanes x dataH x dataW floats) onto the FFT
 * plane (nplanes x fftH x fftW) with the clamp-to-border padding the views
 * receive, values below floor_value raised to it (RL's multiplicative update
 * needs a positive estimate): the initial estimate of a warm start. */
int fmvd_b200_pad_estimate(const fmvd_b200_plan *plan, const float *d_in, float *d_out, int nplanes,
                           float floor_value, void *stream);
/* Convergence check: per plane p of nplanes H x W float planes, in FP64 over
 * rows < rows and columns < cols, d_stats[4p..4p+3] = sum a, sum a^2,
 * sum (a - b)^2, sum |a - b| (d_b may be null: the last two are 0).
 * Deterministic (fixed reduction order). */
int fmvd_b200_plane_stats(const float *d_a, const float *d_b, int nplanes, int H, int W, int rows, int cols,
                          double *d_stats, void *stream);
/* Synchronises with the device and reports whether any kernel of the plan
 * gave up waiting for a bulk copy (bounded waits never hang the GPU; a
 * timeout is reported here as an error). */
int fmvd_b200_plan_check(fmvd_b200_plan *plan);
void fmvd_b200_plan_destroy(fmvd_b200_plan *plan);
/* No counterpart in the reference.  fmvd_b200_deconvolve_device for callers
 * that cannot call cudaMalloc where they deconvolve (a framework's memory pool
 * owns the free device memory, a real-time loop must not take the
 * allocator's device-wide synchronisation, a plugin runs in another
 * application's context): the work planes come from one fixed 64 MiB device
 * array of the library, shared by all plans, instead of the plan's own
 * buffers (which the plan still holds from its creation).  Runs as many plane
 * pairs per batch as fit (at most the plan's batch); a padded plane above
 * about 4.19 M points (2048 x 2048) is rejected with an error.  Call with the
 * plan's device current.  The first call on a device may load the library's
 * module there; make it before any stream capture.  Waits for the stream
 * (also after a failure) and reports a timed-out bulk-copy wait itself.
 * Calls that overlap in time on one device race on the shared array:
 * serialise them. */
int fmvd_b200_deconvolve_device_noalloc(fmvd_b200_plan *plan, const void *d_views, size_t view_stride, void *d_out,
                                        int nplanes, int iterations, float *d_estimate, void *stream);

/* ---- many volumes in one graph launch ------------------------------------ */
/* Captures, once, the deconvolution of 'count' device-resident volumes
 * (volume i: plans[i], d_views[i] with view_strides[i], d_outs[i],
 * nplanes[i] planes, iterations[i]) into one CUDA graph with up to
 * max_branches concurrent branches (0 = 1), balanced by estimated work.
 * Volumes that share a plan run in order on one branch.  Each branch keeps
 * its current batch resident in L2, so more branches only pay for small
 * planes.
 * Buffers must stay valid while the batch exists. */
typedef struct fmvd_b200_batch fmvd_b200_batch;
fmvd_b200_batch *fmvd_b200_batch_create(int count, fmvd_b200_plan *const *plans, const void *const *d_views,
                                        const size_t *view_strides, void *const *d_outs, const int *nplanes,
                                        const int *iterations, int max_branches);
/* One graph launch on stream: every volume of the batch, asynchronously. */
int fmvd_b200_batch_run(fmvd_b200_batch *batch, void *stream);
int fmvd_b200_batch_branches(const fmvd_b200_batch *batch);
void fmvd_b200_batch_destroy(fmvd_b200_batch *batch);

/* Streaming plans with an explicit batch size (the fmvd_initialize_cuda_*
 * entry points choose it automatically). */
struct fmvd_plan_cuda_16 *fmvd_b200_initialize_cuda_16(int dataH, int dataW, float const *const *h_Weights,
                                                       float **h_Kernel, int kernelH, int kernelW,
                                                       fmvd_psf_type iteration_type, int nViews, int nstreams,
                                                       datasource_16_t get_next_plane,
                                                       datasink_16_t return_next_plane, int pairs_per_batch);
struct fmvd_plan_cuda_8 *fmvd_b200_initialize_cuda_8(int dataH, int dataW, float const *const *h_Weights,
                                                     float **h_Kernel, int kernelH, int kernelW,
                                                     fmvd_psf_type iteration_type, int nViews, int nstreams,
                                                     datasource_8_t get_next_plane, datasink_8_t return_next_plane,
                                                     int pairs_per_batch);

/* ---- host buffers in, host buffers out ----------------------------------- */
/* No counterpart in the reference (whose plugin path writes the resampled
 * frame to the host and streams it back plane by plane).  A reconstructor
 * holds the device buffers for one geometry: V source volumes of d planes of
 * h x w samples, a td-plane frame of th x tw (the plan's data plane), work in
 * chunks of chunk_planes target planes (0 = eight plan batches). */
typedef struct fmvd_b200_reconstructor fmvd_b200_reconstructor;
fmvd_b200_reconstructor *fmvd_b200_reconstructor_create(fmvd_b200_plan *plan, int views, int w, int h, int d,
                                                        int tw, int th, int td, int chunk_planes);
/* Resamples view v (h_views[v]: d x h x w contiguous samples, target->source
 * 3x4 matrix h_inverses + 12 v, as transform_cuda_*) into the frame and
 * deconvolves it with the plan (iterations of plain RL); h_out receives td
 * planes of th x tw samples.  The frame never leaves the device; result
 * chunks are copied back while the next chunk computes.  Synchronous;
 * sources in pinned memory upload fastest. */
int fmvd_b200_reconstruct_host(fmvd_b200_reconstructor *rec, const void *const *h_views, const float *h_inverses,
                               int iterations, void *h_out);
void fmvd_b200_reconstructor_destroy(fmvd_b200_reconstructor *rec);

/* ---- resampler ---------------------------------------------------------- */
/* Row pitch (samples) that device source volumes must use. */
size_t fmvd_b200_source_pitch(int bits, int w);
/* Target planes [z0, z0 + nz) from a device source volume (d planes of h
 * rows of 'pitch' samples).  d_out: nz sample planes (or null); d_outf: nz
 * float planes in sample units, before quantisation (or null). */
int fmvd_b200_transform_device(int bits, const void *d_src, size_t pitch, int w, int h, int d, int tw, int th,
                               int z0, int nz, const float *h_inverse, void *d_out, float *d_outf, void *stream);
/* Weight mask of target plane z (tw x th floats). */
int fmvd_b200_mask_device(float *d_out, int z, int w, int h, int d, float zspacing, int tw, int th, float border,
                          const float *h_inverse, void *stream);
/* transform_cuda_* into host memory: h_out receives td planes of tw x th
 * samples (no file, no leading unfilled planes). */
int fmvd_b200_transform_host(int bits, const void *const *h_planes, int w, int h, int d, int tw, int th, int td,
                             const float *h_inverse, void *h_out);

/* ---- tensor-core convolutions of the warm-start network ------------------ */
/* BF16 NHWC activations, weights [cout][taps][cin] (taps 9 = 3 x 3 with zero
 * padding, or 1), FP32 accumulation on the tcgen05 tensor cores:
 * out = relu?(conv(in, weight) + bias + add), zeroed where mask <= 0;
 * d_out (bf16) and/or d_out_f32 receive N x H x W x cout.  cin a multiple of
 * 32, cout a multiple of 16 (at most 256, or a multiple of 256), W a multiple
 * of 8 that divides 128 or is divided by it.  d_status (optional) is set to 1
 * if a wait inside the kernel timed out. */
int fmvd_b200_conv_bf16(const void *d_in, const void *d_weight, int N, int H, int W, int cin, int cout, int taps,
                        void *d_out, float *d_out_f32, const float *d_bias, const void *d_add, const void *d_mask,
                        int relu, int *d_status, void *stream);
/* Weight gradient: d_dw[co][t][ci] += sum over pixels of
 * grad[p][co] * in[p + offset(t)][ci] (FP32, accumulated atomically). */
int fmvd_b200_conv_wgrad_bf16(const void *d_grad, const void *d_in, int N, int H, int W, int cin, int cout, int taps,
                              float *d_dw, int *d_status, void *stream);

/* ---- learned warm start --------------------------------------------------- */
/* A 2-D U-Net (4 levels, base 32 channels, 3 x 3 convolutions, ReLU; BF16
 * weights and activations, FP32 accumulation on the tensor cores) mapping
 * the V registered view planes of a z-plane (uint16, view v of plane z at
 * d_views + v * view_stride + z * H * W) and their mean to an estimate of
 * the plane (float, H x W per plane).  Trained by fmvd_b200_unet_train_step
 * (L1 loss against a target estimate, Adam) on pairs the RL iteration
 * produces; its estimate starts RL through fmvd_b200_pad_estimate and
 * fmvd_b200_deconvolve_device_from.  Planes: height a multiple of 64 (at
 * least 128), width 128, 256, 512 or a multiple of 1024; 1 to 6 views. */
typedef struct fmvd_b200_unet fmvd_b200_unet;
fmvd_b200_unet *fmvd_b200_unet_create(int H, int W, int views, int max_batch, unsigned seed);
void fmvd_b200_unet_destroy(fmvd_b200_unet *net);
/* FP32 parameters, per layer weights [cout][taps][cin] then biases. */
size_t fmvd_b200_unet_param_count(const fmvd_b200_unet *net);
int fmvd_b200_unet_get_params(const fmvd_b200_unet *net, float *h_params);
int fmvd_b200_unet_set_params(fmvd_b200_unet *net, const float *h_params);
/* Gradients of the last training step (lr = 0 computes them without an update). */
int fmvd_b200_unet_get_grads(const fmvd_b200_unet *net, float *h_grads);
/* Estimates of nplanes planes (any count; processed in batches). Asynchronous. */
int fmvd_b200_unet_forward(fmvd_b200_unet *net, const void *d_views, size_t view_stride, int nplanes,
                           float *d_estimate, void *stream);
/* One step on a batch of at most max_batch planes; *h_loss receives the
 * mean L1 loss (in units of the per-plane scale).  Adam with adaptive
 * gradient clipping: a gradient whose L2 norm exceeds twice the running mean
 * of earlier steps' norms is scaled down to it, and a step with a non-finite
 * norm changes nothing.  lr = 0 computes the gradients only.  Synchronous. */
int fmvd_b200_unet_train_step(fmvd_b200_unet *net, const void *d_views, size_t view_stride, int nplanes,
                              const float *d_target, float lr, float *h_loss, void *stream);
/* Synchronises and reports whether a tensor-core wait timed out. */
int fmvd_b200_unet_check(fmvd_b200_unet *net);

/* ---- instrumentation ----------------------------------------------------- */
/* Number of kernel launches the library has issued in this process. */
unsigned long long fmvd_b200_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* FMVD_B200_H */
