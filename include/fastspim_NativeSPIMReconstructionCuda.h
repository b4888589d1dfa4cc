/* JNI entry points of the fastspim Fiji plugin's native class
 * fastspim.NativeSPIMReconstructionCuda (replaces
 * fastspim_NativeSPIMReconstructionCuda.h:11-110 of the reference; same
 * names and Java signatures).  Requires jni.h.
 *
 *   getNumCudaDevices()I, getCudaDeviceName(I)Ljava/lang/String;, setCudaDevice(I)V
 *   transform8/transform16: resample a view (array of per-plane byte[]/short[])
 *   deconvolve: file-based deconvolution (fmvd_deconvolve_files_cuda_*)
 *   deconvolve_init / deconvolve_interactive8/16 / deconvolve_quit8/16:
 *       streaming deconvolution with the Java static callbacks
 *       getNextPlane()[Ljava/lang/Object; and returnNextPlane(Ljava/lang/Object;)V
 */
#ifndef FASTSPIM_NATIVE_SPIM_RECONSTRUCTION_CUDA_H
#define FASTSPIM_NATIVE_SPIM_RECONSTRUCTION_CUDA_H

#include <jni.h>

#ifdef __cplusplus
extern "C" {
#endif

JNIEXPORT jint JNICALL Java_fastspim_NativeSPIMReconstructionCuda_getNumCudaDevices(JNIEnv *env, jclass);

JNIEXPORT jstring JNICALL Java_fastspim_NativeSPIMReconstructionCuda_getCudaDeviceName(JNIEnv *env, jclass,
                                                                                        jint deviceIdx);

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_setCudaDevice(JNIEnv *env, jclass, jint deviceIdx);

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_transform8(
    JNIEnv *env, jclass, jobjectArray data, jint w, jint h, jint d, jfloatArray invMatrix, jint targetW, jint targetH,
    jint targetD, jstring outfile, jboolean createTransformedMasks, jint border, jfloat zspacing, jstring maskfile);

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_transform16(
    JNIEnv *env, jclass, jobjectArray data, jint w, jint h, jint d, jfloatArray invMatrix, jint targetW, jint targetH,
    jint targetD, jstring outfile, jboolean createTransformedMasks, jint border, jfloat zspacing, jstring maskfile);

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve(
    JNIEnv *env, jclass, jobjectArray inputfiles, jstring outputfile, jint dataW, jint dataH, jint dataD,
    jobjectArray weightfiles, jobjectArray kernelfiles, jint kernelH, jint kernelW, jint psfType, jint nViews,
    jint iterations, jint bitDepth);

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1quit8(JNIEnv *env, jclass clazz);

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1quit16(JNIEnv *env, jclass clazz);

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1interactive8(JNIEnv *env, jclass clazz,
                                                                                         jint iterations);

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1interactive16(JNIEnv *env, jclass clazz,
                                                                                          jint iterations);

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1init(
    JNIEnv *env, jclass clazz, jint dataW, jint dataH, jint dataD, jobjectArray weightfiles, jobjectArray kernelfiles,
    jint kernelH, jint kernelW, jint iterationType, jint nViews, jint bitDepth);

#ifdef __cplusplus
}
#endif

#endif
