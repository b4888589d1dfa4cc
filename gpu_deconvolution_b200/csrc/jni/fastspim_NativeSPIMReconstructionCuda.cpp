// JNI binding of the fastspim plugin's native class over the library's C API
// (replaces fastspim_NativeSPIMReconstructionCuda.cpp of the reference).
//
// Behaviour kept from the reference:
//  - every entry installs an error handler that throws java.lang.RuntimeException
//    in the calling JVM thread (fastspim_NativeSPIMReconstructionCuda.cpp:13-24);
//  - deconvolve() selects device 0 (:189), reads kernel and weight files,
//    and runs the file-based deconvolution; bit depths other than 8 and 16 throw;
//  - deconvolve_init() keeps at most one streaming plan per bit depth, with
//    nstreams = min(dataD, 3) (:482), and feeds planes from the static Java
//    methods getNextPlane() (an Object[] of per-view byte[]/short[], or null
//    when done) and returnNextPlane(Object) (:323-377);
//  - deconvolve_quit*() throws when no plan exists.
// Local references created per plane are released after use, so long
// volumes do not exhaust the JVM's local reference table.
#include <jni.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fastspim_NativeSPIMReconstructionCuda.h"
#include "fmvd_cuda_utils.h"
#include "fmvd_deconvolve.h"
#include "fmvd_transform.h"

namespace {

void throw_runtime(void *env_ptr, const char *message)
{
    JNIEnv *env = (JNIEnv *)env_ptr;
    jclass cl = env->FindClass("java/lang/RuntimeException");
    if (cl)
        env->ThrowNew(cl, message);
}

void install_handler(JNIEnv *env) { setErrorHandler(throw_runtime, env); }

// Reads 'count' floats per file for n files named by a Java String[].
bool read_float_files(JNIEnv *env, jobjectArray paths, int n, size_t count, float **dst)
{
    for (int v = 0; v < n; v++) {
        jstring jpath = (jstring)env->GetObjectArrayElement(paths, v);
        const char *path = env->GetStringUTFChars(jpath, NULL);
        FILE *f = fopen(path, "rb");
        bool ok = f && fread(dst[v], sizeof(float), count, f) == count;
        if (f)
            fclose(f);
        if (!ok) {
            char msg[512];
            snprintf(msg, sizeof(msg), "could not read %zu floats from %s", count, path);
            env->ReleaseStringUTFChars(jpath, path);
            env->DeleteLocalRef(jpath);
            throw_runtime(env, msg);
            return false;
        }
        env->ReleaseStringUTFChars(jpath, path);
        env->DeleteLocalRef(jpath);
    }
    return true;
}

struct HostInputs {
    float **kernels = nullptr;
    float **weights = nullptr;
    int n = 0;
    bool load(JNIEnv *env, jobjectArray kernelfiles, jobjectArray weightfiles, int nViews, int kernelH, int kernelW,
              int dataW, int dataH)
    {
        n = nViews;
        kernels = (float **)calloc(n, sizeof(float *));
        weights = (float **)calloc(n, sizeof(float *));
        for (int v = 0; v < n; v++) {
            kernels[v] = (float *)fmvd_malloc((size_t)kernelW * kernelH * sizeof(float));
            weights[v] = (float *)malloc((size_t)dataW * dataH * sizeof(float));
        }
        return read_float_files(env, kernelfiles, n, (size_t)kernelW * kernelH, kernels) &&
               read_float_files(env, weightfiles, n, (size_t)dataW * dataH, weights);
    }
    ~HostInputs()
    {
        for (int v = 0; v < n; v++) {
            fmvd_free(kernels[v]);
            free(weights[v]);
        }
        free(kernels);
        free(weights);
    }
};

// ---- streaming state, one per bit depth (the reference's ia_8 / ia_16)
template <typename S>
struct JavaSide;

template <>
struct JavaSide<unsigned short> {
    typedef jshortArray array_t;
    typedef jshort elem_t;
    typedef fmvd_plan_cuda_16 plan_t;
    static array_t make(JNIEnv *env, jsize n) { return env->NewShortArray(n); }
    static void set(JNIEnv *env, array_t a, jsize n, const unsigned short *src)
    {
        env->SetShortArrayRegion(a, 0, n, (const jshort *)src);
    }
};

template <>
struct JavaSide<unsigned char> {
    typedef jbyteArray array_t;
    typedef jbyte elem_t;
    typedef fmvd_plan_cuda_8 plan_t;
    static array_t make(JNIEnv *env, jsize n) { return env->NewByteArray(n); }
    static void set(JNIEnv *env, array_t a, jsize n, const unsigned char *src)
    {
        env->SetByteArrayRegion(a, 0, n, (const jbyte *)src);
    }
};

template <typename S>
struct Interactive {
    typename JavaSide<S>::plan_t *plan;
    JavaVM *jvm;
    jmethodID get;
    jmethodID put;
    jclass clazz;
    int planesize;
    int nViews;
};

Interactive<unsigned char> *g_ia8 = nullptr;
Interactive<unsigned short> *g_ia16 = nullptr;

template <typename S>
Interactive<S> *&state();
template <>
Interactive<unsigned char> *&state<unsigned char>() { return g_ia8; }
template <>
Interactive<unsigned short> *&state<unsigned short>() { return g_ia16; }

template <typename S>
JNIEnv *attach()
{
    JNIEnv *env = nullptr;
    state<S>()->jvm->AttachCurrentThread((void **)&env, NULL);
    return env;
}

template <typename S>
int get_next_plane(S **data, int offset)
{
    Interactive<S> *ia = state<S>();
    JNIEnv *env = attach<S>();
    jobjectArray arr = (jobjectArray)env->CallStaticObjectMethod(ia->clazz, ia->get);
    if (arr == NULL)
        return 0;
    for (int v = 0; v < ia->nViews; v++) {
        jarray view = (jarray)env->GetObjectArrayElement(arr, v);
        void *src = env->GetPrimitiveArrayCritical(view, NULL);
        memcpy(data[v] + offset, src, (size_t)ia->planesize * sizeof(S));
        env->ReleasePrimitiveArrayCritical(view, src, JNI_ABORT);
        env->DeleteLocalRef(view);
    }
    env->DeleteLocalRef(arr);
    return 1;
}

template <typename S>
void return_next_plane(S *data)
{
    Interactive<S> *ia = state<S>();
    JNIEnv *env = attach<S>();
    typename JavaSide<S>::array_t arr = JavaSide<S>::make(env, ia->planesize);
    JavaSide<S>::set(env, arr, ia->planesize, data);
    env->CallStaticVoidMethod(ia->clazz, ia->put, arr);
    env->DeleteLocalRef(arr);
}

fmvd_plan_cuda_16 *init_plan(unsigned short *, int dataH, int dataW, float **w, float **k, int kH, int kW, int type,
                             int nViews, int nStreams)
{
    return fmvd_initialize_cuda_16(dataH, dataW, w, k, kH, kW, (fmvd_psf_type)type, nViews, nStreams,
                                   get_next_plane<unsigned short>, return_next_plane<unsigned short>);
}

fmvd_plan_cuda_8 *init_plan(unsigned char *, int dataH, int dataW, float **w, float **k, int kH, int kW, int type,
                            int nViews, int nStreams)
{
    return fmvd_initialize_cuda_8(dataH, dataW, w, k, kH, kW, (fmvd_psf_type)type, nViews, nStreams,
                                  get_next_plane<unsigned char>, return_next_plane<unsigned char>);
}

void run_planes(fmvd_plan_cuda_16 *p, int it) { fmvd_deconvolve_planes_cuda_16(p, it); }
void run_planes(fmvd_plan_cuda_8 *p, int it) { fmvd_deconvolve_planes_cuda_8(p, it); }
void destroy_plan(fmvd_plan_cuda_16 *p) { fmvd_destroy_cuda_16(p); }
void destroy_plan(fmvd_plan_cuda_8 *p) { fmvd_destroy_cuda_8(p); }

template <typename S>
void init(JNIEnv *env, jclass clazz, jint dataW, jint dataH, jint dataD, jobjectArray weightfiles,
          jobjectArray kernelfiles, jint kernelH, jint kernelW, jint iterationType, jint nViews)
{
    if (state<S>() != nullptr) {
        throw_runtime(env, "deconvolution already initialized");
        return;
    }
    HostInputs in;
    if (!in.load(env, kernelfiles, weightfiles, nViews, kernelH, kernelW, dataW, dataH))
        return;
    jmethodID get = env->GetStaticMethodID(clazz, "getNextPlane", "()[Ljava/lang/Object;");
    jmethodID put = env->GetStaticMethodID(clazz, "returnNextPlane", "(Ljava/lang/Object;)V");
    if (get == NULL || put == NULL) {
        printf("error in callback: Method not found\n");
        return;
    }
    install_handler(env);
    const int nStreams = dataD < 3 ? dataD : 3;
    auto *plan = init_plan((S *)nullptr, dataH, dataW, in.weights, in.kernels, kernelH, kernelW, iterationType,
                           nViews, nStreams);
    if (!plan)
        return;
    JavaVM *jvm = NULL;
    env->GetJavaVM(&jvm);
    Interactive<S> *ia = new Interactive<S>();
    ia->plan = plan;
    ia->jvm = jvm;
    ia->get = get;
    ia->put = put;
    ia->clazz = (jclass)env->NewGlobalRef(clazz);
    ia->planesize = dataW * dataH;
    ia->nViews = nViews;
    state<S>() = ia;
}

template <typename S>
void interactive(JNIEnv *env, jint iterations)
{
    Interactive<S> *ia = state<S>();
    if (!ia) {
        throw_runtime(env, "deconvolution not initialized");
        return;
    }
    install_handler(env);
    run_planes(ia->plan, iterations);
}

template <typename S>
void quit(JNIEnv *env)
{
    Interactive<S> *ia = state<S>();
    if (!ia) {
        throw_runtime(env, "deconvolution already quit");
        return;
    }
    install_handler(env);
    destroy_plan(ia->plan);
    env->DeleteGlobalRef(ia->clazz);
    delete ia;
    state<S>() = nullptr;
}

template <typename S, typename ArrT, typename ElemT>
void transform(JNIEnv *env, jobjectArray data, jint w, jint h, jint d, jfloatArray invMatrix, jint tw, jint th,
               jint td, jstring outfile, jboolean masks, jint border, jfloat zspacing, jstring maskfile,
               ElemT *(JNIEnv::*get)(ArrT, jboolean *), void (JNIEnv::*rel)(ArrT, ElemT *, jint))
{
    S **planes = (S **)malloc((size_t)d * sizeof(S *));
    ArrT *arrays = (ArrT *)malloc((size_t)d * sizeof(ArrT));
    if (!planes || !arrays) {
        printf("not enough memory\n");
        free(planes);
        free(arrays);
        return;
    }
    for (int z = 0; z < d; z++) {
        arrays[z] = (ArrT)env->GetObjectArrayElement(data, z);
        planes[z] = (S *)(env->*get)(arrays[z], NULL);
    }
    float *mat = env->GetFloatArrayElements(invMatrix, NULL);
    const char *outpath = env->GetStringUTFChars(outfile, NULL);
    const char *maskpath = masks ? env->GetStringUTFChars(maskfile, NULL) : NULL;
    install_handler(env);
    if (sizeof(S) == 2)
        transform_cuda_16((unsigned short **)planes, w, h, d, tw, th, td, mat, outpath, masks, border, zspacing,
                          maskpath);
    else
        transform_cuda_8((unsigned char **)planes, w, h, d, tw, th, td, mat, outpath, masks, border, zspacing,
                         maskpath);
    for (int z = 0; z < d; z++) {
        (env->*rel)(arrays[z], (ElemT *)planes[z], JNI_ABORT);
        env->DeleteLocalRef(arrays[z]);
    }
    env->ReleaseFloatArrayElements(invMatrix, mat, JNI_ABORT);
    env->ReleaseStringUTFChars(outfile, outpath);
    if (masks)
        env->ReleaseStringUTFChars(maskfile, maskpath);
    free(planes);
    free(arrays);
}

} // namespace

extern "C" {

JNIEXPORT jint JNICALL Java_fastspim_NativeSPIMReconstructionCuda_getNumCudaDevices(JNIEnv *env, jclass)
{
    install_handler(env);
    return getNumCUDADevices();
}

JNIEXPORT jstring JNICALL Java_fastspim_NativeSPIMReconstructionCuda_getCudaDeviceName(JNIEnv *env, jclass,
                                                                                        jint deviceIdx)
{
    char name[256] = {0};
    install_handler(env);
    getCudaDeviceName(deviceIdx, name);
    return env->NewStringUTF(name);
}

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_setCudaDevice(JNIEnv *env, jclass, jint deviceIdx)
{
    install_handler(env);
    setCudaDevice(deviceIdx);
}

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_transform16(
    JNIEnv *env, jclass, jobjectArray data, jint w, jint h, jint d, jfloatArray invMatrix, jint targetW, jint targetH,
    jint targetD, jstring outfile, jboolean masks, jint border, jfloat zspacing, jstring maskfile)
{
    transform<unsigned short, jshortArray, jshort>(env, data, w, h, d, invMatrix, targetW, targetH, targetD, outfile,
                                                   masks, border, zspacing, maskfile, &JNIEnv::GetShortArrayElements,
                                                   &JNIEnv::ReleaseShortArrayElements);
}

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_transform8(
    JNIEnv *env, jclass, jobjectArray data, jint w, jint h, jint d, jfloatArray invMatrix, jint targetW, jint targetH,
    jint targetD, jstring outfile, jboolean masks, jint border, jfloat zspacing, jstring maskfile)
{
    transform<unsigned char, jbyteArray, jbyte>(env, data, w, h, d, invMatrix, targetW, targetH, targetD, outfile,
                                                masks, border, zspacing, maskfile, &JNIEnv::GetByteArrayElements,
                                                &JNIEnv::ReleaseByteArrayElements);
}

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve(
    JNIEnv *env, jclass, jobjectArray inputfiles, jstring outputfile, jint dataW, jint dataH, jint dataD,
    jobjectArray weightfiles, jobjectArray kernelfiles, jint kernelH, jint kernelW, jint psfType, jint nViews,
    jint iterations, jint bitDepth)
{
    install_handler(env);
    setCudaDevice(0);
    if (bitDepth != 8 && bitDepth != 16) {
        throw_runtime(env, "Unsupported bit depth");
        return;
    }
    HostInputs in;
    if (!in.load(env, kernelfiles, weightfiles, nViews, kernelH, kernelW, dataW, dataH))
        return;
    FILE **files = (FILE **)calloc(nViews, sizeof(FILE *));
    bool ok = true;
    for (int v = 0; v < nViews && ok; v++) {
        jstring jpath = (jstring)env->GetObjectArrayElement(inputfiles, v);
        const char *path = env->GetStringUTFChars(jpath, NULL);
        files[v] = fopen(path, "rb");
        if (!files[v]) {
            char msg[512];
            snprintf(msg, sizeof(msg), "could not open %s", path);
            throw_runtime(env, msg);
            ok = false;
        }
        env->ReleaseStringUTFChars(jpath, path);
        env->DeleteLocalRef(jpath);
    }
    const char *opath = env->GetStringUTFChars(outputfile, NULL);
    FILE *result = ok ? fopen(opath, "wb") : NULL;
    if (ok && !result) {
        throw_runtime(env, "could not open the output file");
        ok = false;
    }
    env->ReleaseStringUTFChars(outputfile, opath);
    if (ok) {
        install_handler(env);
        if (bitDepth == 8)
            fmvd_deconvolve_files_cuda_8(files, result, dataW, dataH, dataD, in.weights, in.kernels, kernelH, kernelW,
                                         (fmvd_psf_type)psfType, nViews, iterations);
        else
            fmvd_deconvolve_files_cuda_16(files, result, dataW, dataH, dataD, in.weights, in.kernels, kernelH,
                                          kernelW, (fmvd_psf_type)psfType, nViews, iterations);
    }
    for (int v = 0; v < nViews; v++)
        if (files[v])
            fclose(files[v]);
    if (result)
        fclose(result);
    free(files);
}

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1quit8(JNIEnv *env, jclass)
{
    quit<unsigned char>(env);
}

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1quit16(JNIEnv *env, jclass)
{
    quit<unsigned short>(env);
}

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1interactive8(JNIEnv *env, jclass,
                                                                                         jint iterations)
{
    interactive<unsigned char>(env, iterations);
}

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1interactive16(JNIEnv *env, jclass,
                                                                                          jint iterations)
{
    interactive<unsigned short>(env, iterations);
}

JNIEXPORT void JNICALL Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1init(
    JNIEnv *env, jclass clazz, jint dataW, jint dataH, jint dataD, jobjectArray weightfiles, jobjectArray kernelfiles,
    jint kernelH, jint kernelW, jint iterationType, jint nViews, jint bitDepth)
{
    switch (bitDepth) {
    case 8:
        init<unsigned char>(env, clazz, dataW, dataH, dataD, weightfiles, kernelfiles, kernelH, kernelW,
                            iterationType, nViews);
        break;
    case 16:
        init<unsigned short>(env, clazz, dataW, dataH, dataD, weightfiles, kernelfiles, kernelH, kernelW,
                             iterationType, nViews);
        break;
    default:
        throw_runtime(env, "Unsupported bit depth");
    }
}

} // extern "C"
