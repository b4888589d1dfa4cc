/* Minimal stand-in for the JDK's jni.h, for tests only: no JDK exists in this
 * environment.  It declares the subset of the JNI interface (types, JNIEnv
 * and JavaVM member functions, constants) that the library's JNI layer uses,
 * with the JNI specification's names and signatures, so that the same
 * source compiles against the real header.  The member functions are
 * implemented by tests/jni/mock_jvm.cpp, which emulates the Java side. */
#ifndef FMVD_TEST_MOCK_JNI_H
#define FMVD_TEST_MOCK_JNI_H

#include <stdarg.h>
#include <stdint.h>

#define JNIEXPORT __attribute__((visibility("default")))
#define JNICALL
#define JNI_FALSE 0
#define JNI_TRUE 1
#define JNI_COMMIT 1
#define JNI_ABORT 2
#define JNI_OK 0

typedef int32_t jint;
typedef int64_t jlong;
typedef int8_t jbyte;
typedef uint8_t jboolean;
typedef uint16_t jchar;
typedef int16_t jshort;
typedef float jfloat;
typedef double jdouble;
typedef jint jsize;

class _jobject {};
class _jclass : public _jobject {};
class _jstring : public _jobject {};
class _jarray : public _jobject {};
class _jobjectArray : public _jarray {};
class _jshortArray : public _jarray {};
class _jbyteArray : public _jarray {};
class _jfloatArray : public _jarray {};
typedef _jobject *jobject;
typedef _jclass *jclass;
typedef _jstring *jstring;
typedef _jarray *jarray;
typedef _jobjectArray *jobjectArray;
typedef _jshortArray *jshortArray;
typedef _jbyteArray *jbyteArray;
typedef _jfloatArray *jfloatArray;
struct _jmethodID;
typedef _jmethodID *jmethodID;

struct JavaVM_;
typedef JavaVM_ JavaVM;

struct JNIEnv_ {
    jclass FindClass(const char *name);
    jint ThrowNew(jclass clazz, const char *msg);
    jstring NewStringUTF(const char *utf);
    const char *GetStringUTFChars(jstring str, jboolean *isCopy);
    void ReleaseStringUTFChars(jstring str, const char *chars);
    jobject GetObjectArrayElement(jobjectArray array, jsize index);
    jshort *GetShortArrayElements(jshortArray array, jboolean *isCopy);
    void ReleaseShortArrayElements(jshortArray array, jshort *elems, jint mode);
    jbyte *GetByteArrayElements(jbyteArray array, jboolean *isCopy);
    void ReleaseByteArrayElements(jbyteArray array, jbyte *elems, jint mode);
    jfloat *GetFloatArrayElements(jfloatArray array, jboolean *isCopy);
    void ReleaseFloatArrayElements(jfloatArray array, jfloat *elems, jint mode);
    void *GetPrimitiveArrayCritical(jarray array, jboolean *isCopy);
    void ReleasePrimitiveArrayCritical(jarray array, void *carray, jint mode);
    jshortArray NewShortArray(jsize len);
    void SetShortArrayRegion(jshortArray array, jsize start, jsize len, const jshort *buf);
    jbyteArray NewByteArray(jsize len);
    void SetByteArrayRegion(jbyteArray array, jsize start, jsize len, const jbyte *buf);
    jmethodID GetStaticMethodID(jclass clazz, const char *name, const char *sig);
    jobject CallStaticObjectMethod(jclass clazz, jmethodID methodID, ...);
    void CallStaticVoidMethod(jclass clazz, jmethodID methodID, ...);
    jint GetJavaVM(JavaVM **vm);
    jobject NewGlobalRef(jobject obj);
    void DeleteGlobalRef(jobject obj);
    void DeleteLocalRef(jobject obj);
};
typedef JNIEnv_ JNIEnv;

struct JavaVM_ {
    jint AttachCurrentThread(void **penv, void *args);
};

#endif
