// Test-infrastructure restatement of the reference resampler on the hardware
// texture unit (oracle/_ref/libfmvd_reftex.so).  Only the tests, the golden
// fixture generator and bench.py's reference leg load it.
//
// The reference kernel (fmvd_transform.impl.cu:22-56, texture set-up
// :120-128) binds a legacy texture reference, which CUDA 12 removed, so the
// upstream file does not compile here.  This file expresses the same fetch with
// a texture object carrying the same sampler state: unnormalised coordinates,
// linear filtering, border address mode (0 outside) on all three axes and
// normalised-float reads.  The per-voxel arithmetic is the reference's:
// r = M (x, y, z, 1), v = tex3D(r + 0.5), out = (SAMPLE)(v * 2^bits + 0.5).
// It also restates the reference's weight-mask kernel, so that the reference
// arm of the benchmark computes its weights without this project's library.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

namespace {

template <typename S, int BITS>
__global__ void tex_plane_kernel(cudaTextureObject_t tex, S *out, float *raw, int z, int tw, int th,
                                 const float *__restrict__ m)
{
    int x = threadIdx.x + blockIdx.x * blockDim.x;
    int y = threadIdx.y + blockIdx.y * blockDim.y;
    if (x < tw && y < th) {
        float rx = m[0] * x + m[1] * y + m[2] * z + m[3];
        float ry = m[4] * x + m[5] * y + m[6] * z + m[7];
        float rz = m[8] * x + m[9] * y + m[10] * z + m[11];
        float v = tex3D<float>(tex, rx + 0.5, ry + 0.5, rz + 0.5);
        size_t idx = (size_t)y * tw + x;
        if (raw)
            raw[idx] = v;
        out[idx] = (S)(v * (1 << BITS) + 0.5);
    }
}

// Weight mask of target plane z: the reference's create_transformed_mask_kernel
// (fmvd_transform.cu:19-67) -- 0 where the inverse map leaves the source box,
// else the product of the cosine ramps 0.5 (1 - cos(pi dist / border)) of the
// axes nearer than border to an edge, the z distance scaled by zspacing.
__global__ void mask_plane_kernel(float *out, int z, int w, int h, int d, float zspacing, int tw, int th,
                                  float border, const float *__restrict__ m)
{
    const int x = threadIdx.x + blockIdx.x * blockDim.x;
    const int y = threadIdx.y + blockIdx.y * blockDim.y;
    if (x >= tw || y >= th)
        return;
    const float r[3] = {m[0] * x + m[1] * y + m[2] * z + m[3], m[4] * x + m[5] * y + m[6] * z + m[7],
                        m[8] * x + m[9] * y + m[10] * z + m[11]};
    const int ext[3] = {w, h, d};
    float v = 1.f;
    for (int a = 0; a < 3; a++) {
        if (r[a] < 0 || r[a] >= ext[a]) {
            v = 0.f;
            break;
        }
        float dist = r[a] < ext[a] / 2 ? r[a] : ext[a] - r[a];
        if (a == 2)
            dist *= zspacing;
        if (dist < border)
            v *= 0.5f * (1 - cos(dist / border * 3.14159265358979323846f));
    }
    out[(size_t)y * tw + x] = v;
}

// Texture fetch at explicit coordinates (calibration of the filtering model).
__global__ void tex_probe_kernel(cudaTextureObject_t tex, const float *coords, float *vals, int n)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i < n)
        vals[i] = tex3D<float>(tex, coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
}

template <typename S>
cudaTextureObject_t make_texture(const S *h_vol, int w, int h, int d, cudaArray_t *arr_out)
{
    cudaChannelFormatDesc desc = cudaCreateChannelDesc<S>();
    cudaArray_t arr;
    cudaMalloc3DArray(&arr, &desc, make_cudaExtent(w, h, d));
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr((void *)h_vol, w * sizeof(S), w, h);
    p.dstArray = arr;
    p.extent = make_cudaExtent(w, h, d);
    p.kind = cudaMemcpyHostToDevice;
    cudaMemcpy3D(&p);
    cudaResourceDesc res = {};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeNormalizedFloat;
    td.normalizedCoords = 0;
    cudaTextureObject_t tex = 0;
    cudaCreateTextureObject(&tex, &res, &td, NULL);
    *arr_out = arr;
    return tex;
}

template <typename S, int BITS>
int run_transform(const S *h_vol, int w, int h, int d, int tw, int th, int td, const float *h_inv,
                  S *h_out, float *h_raw, float *ms)
{
    cudaArray_t arr;
    cudaTextureObject_t tex = make_texture<S>(h_vol, w, h, d, &arr);
    S *d_out;
    float *d_raw = NULL, *d_m;
    size_t plane = (size_t)tw * th;
    cudaMalloc(&d_out, plane * td * sizeof(S));
    if (h_raw)
        cudaMalloc(&d_raw, plane * td * sizeof(float));
    cudaMalloc(&d_m, 12 * sizeof(float));
    cudaMemcpy(d_m, h_inv, 12 * sizeof(float), cudaMemcpyHostToDevice);
    dim3 threads(32, 32);
    dim3 grid((tw + 31) / 32, (th + 31) / 32);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int z = 0; z < td; z++)
        tex_plane_kernel<S, BITS><<<grid, threads>>>(tex, d_out + plane * z, d_raw ? d_raw + plane * z : NULL,
                                                    z, tw, th, d_m);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    if (ms)
        cudaEventElapsedTime(ms, e0, e1);
    cudaMemcpy(h_out, d_out, plane * td * sizeof(S), cudaMemcpyDeviceToHost);
    if (h_raw)
        cudaMemcpy(h_raw, d_raw, plane * td * sizeof(float), cudaMemcpyDeviceToHost);
    cudaDestroyTextureObject(tex);
    cudaFreeArray(arr);
    cudaFree(d_out);
    cudaFree(d_raw);
    cudaFree(d_m);
    cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? 0 : (int)err;
}

} // namespace

extern "C" {

// Resample a d x h x w volume into td x th x tw with the hardware texture
// path.  h_raw (optional) receives the filtered float before quantisation.
// ms (optional) receives the device time of the plane launches.
int reftex_transform(int bits, const void *h_vol, int w, int h, int d, int tw, int th, int td,
                     const float *h_inv, void *h_out, float *h_raw, float *ms)
{
    if (bits == 16)
        return run_transform<unsigned short, 16>((const unsigned short *)h_vol, w, h, d, tw, th, td, h_inv,
                                                 (unsigned short *)h_out, h_raw, ms);
    return run_transform<unsigned char, 8>((const unsigned char *)h_vol, w, h, d, tw, th, td, h_inv,
                                           (unsigned char *)h_out, h_raw, ms);
}

// Transformed mask of target plane z into h_out (th x tw floats).
int reftex_mask(const float *h_inv, int z, int w, int h, int d, float zspacing, int tw, int th, float border,
                float *h_out)
{
    float *d_out, *d_m;
    cudaMalloc(&d_out, (size_t)tw * th * sizeof(float));
    cudaMalloc(&d_m, 12 * sizeof(float));
    cudaMemcpy(d_m, h_inv, 12 * sizeof(float), cudaMemcpyHostToDevice);
    dim3 threads(32, 32);
    dim3 grid((tw + 31) / 32, (th + 31) / 32);
    mask_plane_kernel<<<grid, threads>>>(d_out, z, w, h, d, zspacing, tw, th, border, d_m);
    cudaMemcpy(h_out, d_out, (size_t)tw * th * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d_out);
    cudaFree(d_m);
    cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? 0 : (int)err;
}

// Hardware texture value at n explicit (x, y, z) coordinates.
int reftex_probe(int bits, const void *h_vol, int w, int h, int d, const float *h_coords, float *h_vals, int n)
{
    cudaArray_t arr;
    cudaTextureObject_t tex = bits == 16 ? make_texture<unsigned short>((const unsigned short *)h_vol, w, h, d, &arr)
                                         : make_texture<unsigned char>((const unsigned char *)h_vol, w, h, d, &arr);
    float *d_c, *d_v;
    cudaMalloc(&d_c, 3 * (size_t)n * sizeof(float));
    cudaMalloc(&d_v, (size_t)n * sizeof(float));
    cudaMemcpy(d_c, h_coords, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
    tex_probe_kernel<<<(n + 255) / 256, 256>>>(tex, d_c, d_v, n);
    cudaMemcpy(h_vals, d_v, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaDestroyTextureObject(tex);
    cudaFreeArray(arr);
    cudaFree(d_c);
    cudaFree(d_v);
    cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? 0 : (int)err;
}

} // extern "C"
