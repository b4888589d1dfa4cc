// Plan objects and the plane-streaming driver behind the public deconvolution
// API (fmvd_initialize / deconvolve_planes / destroy, files entry point).
//
// The reference streams one plane per CUDA stream slot through a ring of
// nstreams slots, 8 launches per view and iteration
// (fmvd_deconvolve.impl.cpp:205-300).  Here planes are gathered into batches
// of 2 * pairs_cap planes (pinned host buffers, three batch slots), copied
// with one transfer per view and direction, and deconvolved together by the
// engine.  Batches alternate between the engine's two lanes (work planes and
// stream each), so consecutive batches also overlap on the device.  While
// batches compute, the host hands the oldest finished batch to the datasink
// and pulls the next one from the datasource into its slot, so host I/O
// overlaps the device work; uploads and downloads run on their own streams.
// The pinned batch buffers outlive their plan in a process-wide pool, so a
// caller that creates one plan per volume (as the plugin does) pins host
// memory once.
#include "fmvd_internal.h"

#include <stdlib.h>
#include <string.h>
#include <mutex>
#include <utility>
#include <vector>

namespace fmvd {

namespace {

// Pinned host buffers released by streaming plans, for later plans of the
// process: pinning (and unpinning) tens of MB takes tens of ms, longer than
// a small volume's whole deconvolution.  At most kPoolBytes stay cached;
// buffers that a device reset released are dropped when found.
constexpr size_t kPoolBytes = size_t(1) << 30;
std::mutex g_pool_lock;
std::vector<std::pair<size_t, void *>> g_pool;  // (bytes, buffer)
size_t g_pool_total = 0;

void *pinned_acquire(size_t bytes)
{
    {
        std::lock_guard<std::mutex> lk(g_pool_lock);
        int best = -1;
        for (int i = 0; i < (int)g_pool.size(); i++) {
            if (!pinned_still_valid(g_pool[i].second)) {  // released by a device reset: forget it
                g_pool_total -= g_pool[i].first;
                g_pool.erase(g_pool.begin() + i--);
                continue;
            }
            if (g_pool[i].first >= bytes && (best < 0 || g_pool[i].first < g_pool[best].first))
                best = i;
        }
        if (best >= 0) {
            void *p = g_pool[best].second;
            g_pool_total -= g_pool[best].first;
            g_pool.erase(g_pool.begin() + best);
            return p;
        }
    }
    void *p = nullptr;
    return FMVD_CHECK(cudaMallocHost(&p, bytes)) ? p : nullptr;
}

void pinned_release(void *p, size_t bytes)
{
    if (!p)
        return;
    {
        std::lock_guard<std::mutex> lk(g_pool_lock);
        if (g_pool_total + bytes <= kPoolBytes) {
            g_pool.emplace_back(bytes, p);
            g_pool_total += bytes;
            return;
        }
    }
    cudaFreeHost(p);
}

template <typename S>
struct Traits;
template <>
struct Traits<unsigned short> {
    using plan_t = fmvd_plan_cuda_16;
    using source_t = datasource_16_t;
    using sink_t = datasink_16_t;
    static constexpr int bits = 16;
};
template <>
struct Traits<unsigned char> {
    using plan_t = fmvd_plan_cuda_8;
    using source_t = datasource_8_t;
    using sink_t = datasink_8_t;
    static constexpr int bits = 8;
};

// FMVD_STRICT_READ_AHEAD=1 in the environment: streaming plans read ahead
// no further than the reference (nstreams planes before the first datasink
// call), for datasources that cannot deliver a plane before earlier ones were
// returned; one batch of at most nstreams planes is in flight at a time.
bool strict_read_ahead()
{
    const char *v = getenv("FMVD_STRICT_READ_AHEAD");
    return v && v[0] && v[0] != '0';
}

template <typename S>
struct Streamer {
    // Three batch slots over the engine's two lanes: batch b fills slot
    // b % 3 and computes on lane b % 2, so while the host fills one slot the
    // two other batches can be computing on both lanes.
    static constexpr int kSlots = 3;
    Engine *eng = nullptr;
    int cap_planes = 0;
    int nslots = kSlots;  // 1 in the strict read-ahead mode
    size_t plane = 0;
    struct Slot {
        S *h_in = nullptr, *d_in = nullptr, *h_out = nullptr, *d_out = nullptr;
        size_t in_bytes = 0, out_bytes = 0;
        std::vector<S *> view_ptrs;
        int n = 0;       // planes of the batch held (0: free)
        cudaEvent_t up = nullptr, done = nullptr, down = nullptr;
    } slot[kSlots];
    Engine lane[2];              // the engine with each lane's work planes
    cudaStream_t comp[2] = {nullptr, nullptr};
    int nlanes = 1;
    cudaStream_t s_up = nullptr, s_down = nullptr;

    bool init(Engine *e, int nstreams)
    {
        eng = e;
        cap_planes = 2 * e->pairs_cap;
        if (strict_read_ahead()) {
            // the datasource runs at most nstreams planes (and at most one
            // batch) ahead of the datasink, as in the reference
            nslots = 1;
            cap_planes = nstreams < cap_planes ? nstreams : cap_planes;
        }
        plane = (size_t)e->dims.dataH * e->dims.dataW;
        const int V = e->dims.V;
        nlanes = e->lanes > 1 ? 2 : 1;
        lane[0] = lane[1] = *e;
        if (nlanes > 1) {
            lane[1].C = e->laneC[0];
            lane[1].est = e->laneEst[0];
        }
        bool ok = FMVD_CHECK(cudaStreamCreateWithFlags(&s_up, cudaStreamNonBlocking)) &&
                  FMVD_CHECK(cudaStreamCreateWithFlags(&s_down, cudaStreamNonBlocking));
        for (int l = 0; l < nlanes && ok; l++)
            ok = FMVD_CHECK(cudaStreamCreateWithFlags(&comp[l], cudaStreamNonBlocking));
        for (int k = 0; k < nslots && ok; k++) {
            Slot &sl = slot[k];
            const size_t in_bytes = sizeof(S) * plane * cap_planes * V;
            const size_t out_bytes = sizeof(S) * plane * cap_planes;
            sl.h_in = (S *)pinned_acquire(in_bytes);
            sl.in_bytes = sl.h_in ? in_bytes : 0;
            sl.h_out = sl.h_in ? (S *)pinned_acquire(out_bytes) : nullptr;
            sl.out_bytes = sl.h_out ? out_bytes : 0;
            ok = sl.h_in && sl.h_out && FMVD_CHECK(cudaMalloc(&sl.d_in, in_bytes)) &&
                 FMVD_CHECK(cudaMalloc(&sl.d_out, out_bytes)) &&
                 FMVD_CHECK(cudaEventCreateWithFlags(&sl.up, cudaEventDisableTiming)) &&
                 FMVD_CHECK(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) &&
                 FMVD_CHECK(cudaEventCreateWithFlags(&sl.down, cudaEventDisableTiming));
            if (ok) {  // no clearing: only planes the datasource wrote are uploaded
                sl.view_ptrs.resize(V);
                for (int v = 0; v < V; v++)
                    sl.view_ptrs[v] = sl.h_in + (size_t)v * cap_planes * plane;
            }
        }
        return ok;
    }

    void release()
    {
        for (auto &sl : slot) {
            pinned_release(sl.h_in, sl.in_bytes);
            cudaFree(sl.d_in);
            pinned_release(sl.h_out, sl.out_bytes);
            cudaFree(sl.d_out);
            if (sl.up) cudaEventDestroy(sl.up);
            if (sl.done) cudaEventDestroy(sl.done);
            if (sl.down) cudaEventDestroy(sl.down);
        }
        for (cudaStream_t c : comp)
            if (c)
                cudaStreamDestroy(c);
        if (s_up) cudaStreamDestroy(s_up);
        if (s_down) cudaStreamDestroy(s_down);
    }
};

template <typename S>
struct Plan {
    typename Traits<S>::plan_t pub;  // first member: the public struct
    Streamer<S> st;
};

template <typename S>
typename Traits<S>::plan_t *initialize(int dataH, int dataW, const float *const *h_Weights, float **h_Kernel,
                                       int kernelH, int kernelW, int type, int nViews, int nstreams,
                                       typename Traits<S>::source_t src, typename Traits<S>::sink_t sink,
                                       int pairs_cap)
{
    if (nstreams < 1) {
        report_error("fmvd: nstreams must be at least 1");
        return nullptr;
    }
    Engine *e = engine_create(Traits<S>::bits, dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, type, nViews,
                              pairs_cap, 0, 2);
    if (!e)
        return nullptr;
    Plan<S> *p = new Plan<S>();
    if (!p->st.init(e, nstreams)) {
        p->st.release();
        engine_destroy(e);
        delete p;
        return nullptr;
    }
    auto &q = p->pub;
    q.dataH = dataH;
    q.dataW = dataW;
    q.fftH = e->dims.H;
    q.fftW = e->dims.W;
    q.kernelH = kernelH;
    q.kernelW = kernelW;
    q.nViews = nViews;
    q.nStreams = nstreams;
    q.get_next_plane = src;
    q.return_next_plane = sink;
    q.engine = p;
    return &p->pub;
}

template <typename S>
void destroy(typename Traits<S>::plan_t *plan)
{
    if (!plan)
        return;
    Plan<S> *p = reinterpret_cast<Plan<S> *>(plan->engine);
    cudaDeviceSynchronize();
    Engine *e = p->st.eng;
    p->st.release();
    engine_destroy(e);
    delete p;
}

template <typename S>
void deconvolve_planes(const typename Traits<S>::plan_t *plan, int iterations)
{
    if (!plan)
        return;
    Plan<S> *p = reinterpret_cast<Plan<S> *>(plan->engine);
    Streamer<S> &st = p->st;
    Engine *e = st.eng;
    const int V = e->dims.V;
    const size_t plane = st.plane;
    const int cap = st.cap_planes;
    const size_t view_stride = plane * cap;
    auto get = plan->get_next_plane;
    auto put = plan->return_next_plane;

    bool exhausted = false;
    int obtained = 0;  // planes handed out by the source, plus unfilled quirk slots
    // Fill a slot from the datasource.  The reference primes nstreams slots
    // without looking at the return value (fmvd_deconvolve.impl.cpp:216-219),
    // so a source holding fewer planes than nstreams still produces nstreams
    // planes; the extra calls are made here once the source runs dry.
    auto fill = [&](typename Streamer<S>::Slot &sl) {
        sl.n = 0;
        while (sl.n < cap) {
            if (!exhausted) {
                if (get(sl.view_ptrs.data(), (int)(sl.n * plane))) {
                    sl.n++;
                    obtained++;
                    continue;
                }
                exhausted = true;
            }
            if (obtained >= plan->nStreams)
                break;
            for (int v = 0; v < V; v++)
                memset(sl.view_ptrs[v] + sl.n * plane, 0, plane * sizeof(S));
            get(sl.view_ptrs.data(), (int)(sl.n * plane));
            sl.n++;
            obtained++;
        }
    };

    const int K = st.nslots;
    // hands a finished batch to the datasink (planes in z order)
    auto drain = [&](typename Streamer<S>::Slot &sl) -> bool {
        if (sl.n == 0)
            return true;
        if (!FMVD_CHECK(cudaEventSynchronize(sl.down)))
            return false;
        for (int i = 0; i < sl.n; i++)
            put(sl.h_out + (size_t)i * plane);
        sl.n = 0;
        return true;
    };
    int b = 0;
    for (;; b++) {
        auto &sl = st.slot[b % K];
        // the slot's previous batch (b - K), the oldest in flight, goes out first
        if (!drain(sl))
            return;
        fill(sl);
        if (sl.n == 0)
            break;
        // upload: one copy per view (the slot's previous batch has been
        // downloaded, so its device buffers are free)
        for (int v = 0; v < V; v++)
            if (!FMVD_CHECK(cudaMemcpyAsync(sl.d_in + view_stride * v, sl.view_ptrs[v], sizeof(S) * plane * sl.n,
                                            cudaMemcpyHostToDevice, st.s_up)))
                return;
        const int l = b % st.nlanes;
        const cudaStream_t cs = st.comp[l];
        if (!FMVD_CHECK(cudaEventRecord(sl.up, st.s_up)) || !FMVD_CHECK(cudaStreamWaitEvent(cs, sl.up, 0)))
            return;
        engine_batch(&st.lane[l], sl.d_in, view_stride, sl.d_out, sl.n, iterations, cs);
        if (!FMVD_CHECK(cudaGetLastError()) || !FMVD_CHECK(cudaEventRecord(sl.done, cs)) ||
            !FMVD_CHECK(cudaStreamWaitEvent(st.s_down, sl.done, 0)) ||
            !FMVD_CHECK(cudaMemcpyAsync(sl.h_out, sl.d_out, sizeof(S) * plane * sl.n, cudaMemcpyDeviceToHost,
                                        st.s_down)) ||
            !FMVD_CHECK(cudaEventRecord(sl.down, st.s_down)))
            return;
    }
    // the batches still in flight, oldest first
    for (int j = b - K + 1; j < b; j++)
        if (j >= 0 && !drain(st.slot[j % K]))
            return;
    engine_check_status(e);
}

// fmvd_deconvolve_hdd.impl.cpp:16-76: the file source reads one plane per
// view, the file sink writes one plane; nstreams is 3.
template <typename S>
struct FileIO {
    static FILE **files;
    static FILE *result;
    static size_t planesize;
    static int plane, nplanes, nviews;
    static int source(S **data, int offset)
    {
        if (plane >= nplanes)
            return 0;
        for (int v = 0; v < nviews; v++)
            if (fread(data[v] + offset, sizeof(S), planesize, files[v]) != planesize)
                report_error("fmvd: short read from a data file");
        plane++;
        return 1;
    }
    static void sink(S *data) { fwrite(data, sizeof(S), planesize, result); }
};
template <typename S> FILE **FileIO<S>::files = nullptr;
template <typename S> FILE *FileIO<S>::result = nullptr;
template <typename S> size_t FileIO<S>::planesize = 0;
template <typename S> int FileIO<S>::plane = 0;
template <typename S> int FileIO<S>::nplanes = 0;
template <typename S> int FileIO<S>::nviews = 0;

template <typename S>
void deconvolve_files(FILE **dataFiles, FILE *resultFile, int dataW, int dataH, int dataD, float **h_Weights,
                      float **h_Kernel, int kernelH, int kernelW, int type, int nViews, int iterations)
{
    using IO = FileIO<S>;
    IO::files = dataFiles;
    IO::result = resultFile;
    IO::planesize = (size_t)dataW * dataH;
    IO::plane = 0;
    IO::nplanes = dataD;
    IO::nviews = nViews;
    auto *plan = initialize<S>(dataH, dataW, h_Weights, h_Kernel, kernelH, kernelW, type, nViews, 3, IO::source,
                               IO::sink, 0);
    if (!plan)
        return;
    deconvolve_planes<S>(plan, iterations);
    destroy<S>(plan);
}

} // namespace

// ---------------------------------------------------------------- exports
void *pinned_malloc(size_t size)
{
    void *p = nullptr;
    if (!FMVD_CHECK(cudaMallocHost(&p, size)))
        return nullptr;
    return p;
}

void pinned_free(void *p) { cudaFreeHost(p); }

bool pinned_still_valid(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

fmvd_plan_cuda_16 *initialize_16(int dataH, int dataW, const float *const *w, float **k, int kH, int kW, int type,
                                 int V, int nstreams, datasource_16_t src, datasink_16_t sink, int pairs_cap)
{
    return initialize<unsigned short>(dataH, dataW, w, k, kH, kW, type, V, nstreams, src, sink, pairs_cap);
}

fmvd_plan_cuda_8 *initialize_8(int dataH, int dataW, const float *const *w, float **k, int kH, int kW, int type,
                               int V, int nstreams, datasource_8_t src, datasink_8_t sink, int pairs_cap)
{
    return initialize<unsigned char>(dataH, dataW, w, k, kH, kW, type, V, nstreams, src, sink, pairs_cap);
}

void deconvolve_planes_16(const fmvd_plan_cuda_16 *p, int it) { deconvolve_planes<unsigned short>(p, it); }
void deconvolve_planes_8(const fmvd_plan_cuda_8 *p, int it) { deconvolve_planes<unsigned char>(p, it); }
void destroy_16(fmvd_plan_cuda_16 *p) { destroy<unsigned short>(p); }
void destroy_8(fmvd_plan_cuda_8 *p) { destroy<unsigned char>(p); }

void deconvolve_files_16(FILE **f, FILE *r, int dW, int dH, int dD, float **w, float **k, int kH, int kW, int type,
                         int V, int it)
{
    deconvolve_files<unsigned short>(f, r, dW, dH, dD, w, k, kH, kW, type, V, it);
}

void deconvolve_files_8(FILE **f, FILE *r, int dW, int dH, int dD, float **w, float **k, int kH, int kW, int type,
                        int V, int it)
{
    deconvolve_files<unsigned char>(f, r, dW, dH, dD, w, k, kH, kW, type, V, it);
}

Engine *plan_engine_16(const fmvd_plan_cuda_16 *p) { return p ? reinterpret_cast<Plan<unsigned short> *>(p->engine)->st.eng : nullptr; }
Engine *plan_engine_8(const fmvd_plan_cuda_8 *p) { return p ? reinterpret_cast<Plan<unsigned char> *>(p->engine)->st.eng : nullptr; }

} // namespace fmvd
