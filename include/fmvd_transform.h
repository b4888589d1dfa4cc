/* Affine trilinear resampling of a view into the common frame, C ABI.
 *
 * Replaces transform_cuda_8 / transform_cuda_16 (fmvd_transform.h:4-24,
 * fmvd_transform.impl.cu:77-224 of the reference; C++ linkage there, both
 * linkages exported here).  Semantics kept:
 *  - h_data holds d plane pointers, each w x h samples (x fastest);
 *  - h_inverse is the 3 x 4 row-major target -> source matrix;
 *  - each target voxel takes the trilinear interpolation of the source at
 *    M (x, y, z, 1), sampled like a CUDA linear texture with border value 0
 *    (weights quantised to 1/256), normalised by 2^bits - 1 and stored as
 *    (sample)(v * 2^bits + 0.5), saturated;
 *  - outfile receives td planes of tw x th samples (for td == 1 the reference
 *    writes an unfilled plane before plane 0: here a zero plane);
 *  - with createTransformedMasks, maskfile receives the float32 tw x th
 *    weight image of plane td / 2: 0 outside the source box, else the
 *    product over axes of 0.5 (1 - cos(pi d / border)) where the distance d
 *    to the nearest box face (z distance times zspacing) is below border.
 */
#ifndef FMVD_TRANSFORM_H
#define FMVD_TRANSFORM_H

#ifdef __cplusplus
extern "C" {
#endif

void transform_cuda_8(unsigned char **h_data, int w, int h, int d, int tw, int th, int td, float *h_inverse,
                      const char *outfile, int createTransformedMasks, int border, float zspacing,
                      const char *maskfile);

void transform_cuda_16(unsigned short **h_data, int w, int h, int d, int tw, int th, int td, float *h_inverse,
                       const char *outfile, int createTransformedMasks, int border, float zspacing,
                       const char *maskfile);

#ifdef __cplusplus
}
#endif

#endif /* FMVD_TRANSFORM_H */
