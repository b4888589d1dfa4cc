// A tiny emulation of the Java side for the JNI layer tests: Java objects
// are C++ objects owned by the mock, the plugin class has the static
// callbacks getNextPlane() and returnNextPlane(Object), and a driver (main)
// exercises the JNI entry points the Fiji plugin calls.
//
//   jni_driver <bits> <dataW> <dataH> <dataD> <nViews> <kW> <kH> <iterations> <psf>
//              <views.raw> <weights.raw> <kernels.raw> <out_dir>
//
// views.raw: nViews x dataD x dataH x dataW samples; weights.raw: nViews x
// dataH x dataW floats; kernels.raw: nViews x kH x kW floats.  Writes
// out_dir/interactive.raw (planes the plugin received through
// returnNextPlane) and out_dir/files.raw (file-based entry), and prints one
// line per JNI call with the exceptions it raised.
#include <jni.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <memory>
#include <string>
#include <vector>

#include "fastspim_NativeSPIMReconstructionCuda.h"

namespace {

struct Obj : _jobject {
    virtual ~Obj() {}
};
struct ClassObj : Obj {
};
struct StringObj : Obj {
    std::string s;
};
template <typename T>
struct ArrayObj : Obj {
    std::vector<T> v;
};
struct ObjArray : Obj {
    std::vector<jobject> v;
};

std::vector<std::unique_ptr<Obj>> g_heap;
std::vector<std::string> g_exceptions;
int g_live_local = 0;

template <typename T>
T *keep(T *o)
{
    g_heap.emplace_back(o);
    g_live_local++;
    return o;
}

// ---- the plugin class state (Java side)
int g_bits = 16, g_W, g_H, g_D, g_V;
std::vector<char> g_views;      // V x D x H x W samples
size_t g_next = 0;
std::vector<char> g_received;   // planes delivered by returnNextPlane
size_t g_returned = 0;

jobject get_next_plane_java()
{
    if (g_next >= (size_t)g_D)
        return nullptr;
    ObjArray *arr = keep(new ObjArray());
    const size_t plane = (size_t)g_W * g_H;
    const size_t es = g_bits / 8;
    for (int v = 0; v < g_V; v++) {
        const char *src = g_views.data() + ((size_t)v * g_D + g_next) * plane * es;
        if (g_bits == 16) {
            auto *a = keep(new ArrayObj<jshort>());
            a->v.assign((const jshort *)src, (const jshort *)src + plane);
            arr->v.push_back(a);
        } else {
            auto *a = keep(new ArrayObj<jbyte>());
            a->v.assign((const jbyte *)src, (const jbyte *)src + plane);
            arr->v.push_back(a);
        }
    }
    g_next++;
    return arr;
}

void return_next_plane_java(jobject o)
{
    const size_t plane = (size_t)g_W * g_H;
    if (g_bits == 16) {
        auto *a = static_cast<ArrayObj<jshort> *>(static_cast<Obj *>(o));
        g_received.insert(g_received.end(), (char *)a->v.data(), (char *)(a->v.data() + plane));
    } else {
        auto *a = static_cast<ArrayObj<jbyte> *>(static_cast<Obj *>(o));
        g_received.insert(g_received.end(), (char *)a->v.data(), (char *)(a->v.data() + plane));
    }
    g_returned++;
}

JavaVM_ g_vm;
JNIEnv_ g_env;
ClassObj g_plugin_class;
_jmethodID *const kGet = (_jmethodID *)0x1;
_jmethodID *const kPut = (_jmethodID *)0x2;

} // namespace

// ---- JNIEnv / JavaVM member functions
jclass JNIEnv_::FindClass(const char *) { return (jclass)(_jobject *)keep(new ClassObj()); }
jint JNIEnv_::ThrowNew(jclass, const char *msg)
{
    g_exceptions.push_back(msg ? msg : "");
    return 0;
}
jstring JNIEnv_::NewStringUTF(const char *utf)
{
    StringObj *s = keep(new StringObj());
    s->s = utf;
    return (jstring)(_jobject *)s;
}
const char *JNIEnv_::GetStringUTFChars(jstring str, jboolean *) { return ((StringObj *)(_jobject *)str)->s.c_str(); }
void JNIEnv_::ReleaseStringUTFChars(jstring, const char *) {}
jobject JNIEnv_::GetObjectArrayElement(jobjectArray array, jsize index)
{
    g_live_local++;
    return static_cast<ObjArray *>(static_cast<Obj *>((_jobject *)array))->v[index];
}
jshort *JNIEnv_::GetShortArrayElements(jshortArray a, jboolean *)
{
    return static_cast<ArrayObj<jshort> *>(static_cast<Obj *>((_jobject *)a))->v.data();
}
void JNIEnv_::ReleaseShortArrayElements(jshortArray, jshort *, jint) {}
jbyte *JNIEnv_::GetByteArrayElements(jbyteArray a, jboolean *)
{
    return static_cast<ArrayObj<jbyte> *>(static_cast<Obj *>((_jobject *)a))->v.data();
}
void JNIEnv_::ReleaseByteArrayElements(jbyteArray, jbyte *, jint) {}
jfloat *JNIEnv_::GetFloatArrayElements(jfloatArray a, jboolean *)
{
    return static_cast<ArrayObj<jfloat> *>(static_cast<Obj *>((_jobject *)a))->v.data();
}
void JNIEnv_::ReleaseFloatArrayElements(jfloatArray, jfloat *, jint) {}
void *JNIEnv_::GetPrimitiveArrayCritical(jarray a, jboolean *)
{
    Obj *o = static_cast<Obj *>((_jobject *)a);
    if (auto *s = dynamic_cast<ArrayObj<jshort> *>(o))
        return s->v.data();
    if (auto *b = dynamic_cast<ArrayObj<jbyte> *>(o))
        return b->v.data();
    return nullptr;
}
void JNIEnv_::ReleasePrimitiveArrayCritical(jarray, void *, jint) {}
jshortArray JNIEnv_::NewShortArray(jsize len)
{
    auto *a = keep(new ArrayObj<jshort>());
    a->v.resize(len);
    return (jshortArray)(_jobject *)a;
}
void JNIEnv_::SetShortArrayRegion(jshortArray arr, jsize start, jsize len, const jshort *buf)
{
    auto *a = static_cast<ArrayObj<jshort> *>(static_cast<Obj *>((_jobject *)arr));
    memcpy(a->v.data() + start, buf, len * sizeof(jshort));
}
jbyteArray JNIEnv_::NewByteArray(jsize len)
{
    auto *a = keep(new ArrayObj<jbyte>());
    a->v.resize(len);
    return (jbyteArray)(_jobject *)a;
}
void JNIEnv_::SetByteArrayRegion(jbyteArray arr, jsize start, jsize len, const jbyte *buf)
{
    auto *a = static_cast<ArrayObj<jbyte> *>(static_cast<Obj *>((_jobject *)arr));
    memcpy(a->v.data() + start, buf, len);
}
jmethodID JNIEnv_::GetStaticMethodID(jclass, const char *name, const char *sig)
{
    if (!strcmp(name, "getNextPlane") && !strcmp(sig, "()[Ljava/lang/Object;"))
        return kGet;
    if (!strcmp(name, "returnNextPlane") && !strcmp(sig, "(Ljava/lang/Object;)V"))
        return kPut;
    return nullptr;
}
jobject JNIEnv_::CallStaticObjectMethod(jclass, jmethodID m, ...)
{
    return m == kGet ? get_next_plane_java() : nullptr;
}
void JNIEnv_::CallStaticVoidMethod(jclass, jmethodID m, ...)
{
    va_list ap;
    va_start(ap, m);
    jobject o = va_arg(ap, jobject);
    va_end(ap);
    if (m == kPut)
        return_next_plane_java(o);
}
jint JNIEnv_::GetJavaVM(JavaVM **vm)
{
    *vm = &g_vm;
    return JNI_OK;
}
jobject JNIEnv_::NewGlobalRef(jobject o) { return o; }
void JNIEnv_::DeleteGlobalRef(jobject) {}
void JNIEnv_::DeleteLocalRef(jobject) { g_live_local--; }
jint JavaVM_::AttachCurrentThread(void **penv, void *)
{
    *penv = &g_env;
    return JNI_OK;
}

// ---- driver
static std::vector<char> read_file(const char *p)
{
    std::vector<char> d;
    FILE *f = fopen(p, "rb");
    if (!f)
        return d;
    fseek(f, 0, SEEK_END);
    d.resize(ftell(f));
    fseek(f, 0, SEEK_SET);
    if (fread(d.data(), 1, d.size(), f) != d.size())
        d.clear();
    fclose(f);
    return d;
}

static jobjectArray string_array(const std::vector<std::string> &s)
{
    ObjArray *a = keep(new ObjArray());
    for (auto &x : s)
        a->v.push_back(g_env.NewStringUTF(x.c_str()));
    return (jobjectArray)(_jobject *)a;
}

static void report(const char *call)
{
    printf("%s exceptions=%zu", call, g_exceptions.size());
    for (auto &e : g_exceptions)
        printf(" [%s]", e.c_str());
    printf("\n");
    g_exceptions.clear();
}

int main(int argc, char **argv)
{
    JNIEnv *env = &g_env;
    jclass cls = (jclass)(_jobject *)&g_plugin_class;
    if (argc == 2 && !strcmp(argv[1], "errors")) {
        // paths that need no GPU: quitting without a plan, a bad bit depth
        Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1quit16(env, cls);
        report("quit16_without_init");
        Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1quit8(env, cls);
        report("quit8_without_init");
        Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1interactive16(env, cls, 1);
        report("interactive16_without_init");
        Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1init(env, cls, 8, 8, 1, string_array({}),
                                                                    string_array({}), 3, 3, 0, 0, 12);
        report("init_bad_bitdepth");
        return 0;
    }
    if (argc < 14) {
        fprintf(stderr, "usage: see source\n");
        return 2;
    }
    g_bits = atoi(argv[1]);
    g_W = atoi(argv[2]);
    g_H = atoi(argv[3]);
    g_D = atoi(argv[4]);
    g_V = atoi(argv[5]);
    const int kW = atoi(argv[6]), kH = atoi(argv[7]), its = atoi(argv[8]), psf = atoi(argv[9]);
    const std::string views = argv[10], weights = argv[11], kernels = argv[12], out = argv[13];
    g_views = read_file(views.c_str());
    std::vector<char> wts = read_file(weights.c_str()), krn = read_file(kernels.c_str());
    // per-view weight and kernel files, as the plugin passes them
    std::vector<std::string> wfiles, kfiles, vfiles;
    const size_t plane = (size_t)g_W * g_H, es = g_bits / 8;
    for (int v = 0; v < g_V; v++) {
        std::string wf = out + "/w" + std::to_string(v) + ".raw", kf = out + "/k" + std::to_string(v) + ".raw",
                    vf = out + "/v" + std::to_string(v) + ".raw";
        FILE *f = fopen(wf.c_str(), "wb");
        fwrite(wts.data() + v * plane * 4, 4, plane, f);
        fclose(f);
        f = fopen(kf.c_str(), "wb");
        fwrite(krn.data() + (size_t)v * kW * kH * 4, 4, (size_t)kW * kH, f);
        fclose(f);
        f = fopen(vf.c_str(), "wb");
        fwrite(g_views.data() + (size_t)v * g_D * plane * es, es, (size_t)g_D * plane, f);
        fclose(f);
        wfiles.push_back(wf);
        kfiles.push_back(kf);
        vfiles.push_back(vf);
    }
    printf("devices=%d\n", Java_fastspim_NativeSPIMReconstructionCuda_getNumCudaDevices(env, cls));
    report("getNumCudaDevices");
    jstring name = Java_fastspim_NativeSPIMReconstructionCuda_getCudaDeviceName(env, cls, 0);
    printf("name=%s\n", env->GetStringUTFChars(name, nullptr));
    report("getCudaDeviceName");
    Java_fastspim_NativeSPIMReconstructionCuda_setCudaDevice(env, cls, 0);
    report("setCudaDevice");

    // streaming entry points
    Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1init(env, cls, g_W, g_H, g_D, string_array(wfiles),
                                                                string_array(kfiles), kH, kW, psf, g_V, g_bits);
    report("deconvolve_init");
    Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1init(env, cls, g_W, g_H, g_D, string_array(wfiles),
                                                                string_array(kfiles), kH, kW, psf, g_V, g_bits);
    report("deconvolve_init_twice");
    if (g_bits == 16)
        Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1interactive16(env, cls, its);
    else
        Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1interactive8(env, cls, its);
    report("deconvolve_interactive");
    if (g_bits == 16)
        Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1quit16(env, cls);
    else
        Java_fastspim_NativeSPIMReconstructionCuda_deconvolve_1quit8(env, cls);
    report("deconvolve_quit");
    printf("returned=%zu local_refs_live=%d\n", g_returned, g_live_local);
    FILE *f = fopen((out + "/interactive.raw").c_str(), "wb");
    fwrite(g_received.data(), 1, g_received.size(), f);
    fclose(f);

    // file-based entry point
    jstring outp = env->NewStringUTF((out + "/files.raw").c_str());
    Java_fastspim_NativeSPIMReconstructionCuda_deconvolve(env, cls, string_array(vfiles), outp, g_W, g_H, g_D,
                                                          string_array(wfiles), string_array(kfiles), kH, kW, psf,
                                                          g_V, its, g_bits);
    report("deconvolve_files");
    return 0;
}
