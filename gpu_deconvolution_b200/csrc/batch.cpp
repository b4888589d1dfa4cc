// Many independent volumes of uneven plane sizes deconvolved by one CUDA
// graph launch.
//
// Each volume keeps its own plan (spectra, weights, work planes).  At
// creation the launch sequences of all volumes are captured once into one
// graph; the host issues a single graph launch per run instead of thousands
// of kernel launches.  The graph may have several concurrent branches
// (balanced by estimated work); volumes that share a plan share its work
// planes, so they go to the same branch and run in order.  Each plan already
// runs two batch lanes and keeps its batches resident in L2, so concurrent
// branches evict each other: on the 32-volume workload one branch measured
// fastest, and it is the default.
#include "fmvd_b200.h"
#include "fmvd_internal.h"

#include <algorithm>
#include <map>
#include <vector>

struct fmvd_b200_batch {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaStream_t> streams;  // [0] origin of the capture, then one per branch
    std::vector<cudaEvent_t> events;
    int branches = 0;
    unsigned long long kernels = 0;  // kernel nodes captured (added to the launch count per run)
};

namespace {

void release(fmvd_b200_batch *b)
{
    if (!b)
        return;
    if (b->exec)
        cudaGraphExecDestroy(b->exec);
    if (b->graph)
        cudaGraphDestroy(b->graph);
    for (cudaEvent_t e : b->events)
        cudaEventDestroy(e);
    for (cudaStream_t s : b->streams)
        cudaStreamDestroy(s);
    delete b;
}

} // namespace

extern "C" {

fmvd_b200_batch *fmvd_b200_batch_create(int count, fmvd_b200_plan *const *plans, const void *const *d_views,
                                        const size_t *view_strides, void *const *d_outs, const int *nplanes,
                                        const int *iterations, int max_branches)
{
    if (count < 1 || !plans || !d_views || !view_strides || !d_outs || !nplanes || !iterations) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_batch_create");
        return nullptr;
    }
    for (int i = 0; i < count; i++)
        if (!plans[i] || nplanes[i] < 0) {
            fmvd::report_error("fmvd: fmvd_b200_batch_create: missing plan or negative plane count");
            return nullptr;
        }
    if (max_branches < 1)
        max_branches = 1;

    // Branch of each volume: volumes sharing a plan stay together; groups go,
    // largest estimated work first, to the branch with the least work so far
    // (work ~ planes x padded plane x views x iterations).
    std::map<const fmvd_b200_plan *, std::vector<int>> groups;
    for (int i = 0; i < count; i++)
        groups[plans[i]].push_back(i);
    std::vector<std::pair<double, const fmvd_b200_plan *>> order;
    for (auto &g : groups) {
        const fmvd::RlDims &d = g.first->eng->dims;
        double w = 0;
        for (int i : g.second)
            w += (double)nplanes[i] * d.H * d.W * d.V * (iterations[i] > 0 ? iterations[i] : 1);
        order.push_back({w, g.first});
    }
    std::sort(order.begin(), order.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    const int nb = (int)order.size() < max_branches ? (int)order.size() : max_branches;
    std::vector<double> load(nb, 0.0);
    std::vector<int> branch(count);
    for (auto &o : order) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[k] += o.first;
        for (int i : groups[o.second])
            branch[i] = k;
    }

    fmvd_b200_batch *b = new fmvd_b200_batch();
    b->branches = nb;
    bool ok = true;
    for (int i = 0; i <= nb && ok; i++) {
        cudaStream_t s = nullptr;
        ok = FMVD_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        if (ok)
            b->streams.push_back(s);
    }
    for (int i = 0; i <= nb && ok; i++) {
        cudaEvent_t e = nullptr;
        ok = FMVD_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        if (ok)
            b->events.push_back(e);
    }
    if (!ok) {
        release(b);
        return nullptr;
    }

    cudaStream_t origin = b->streams[0];
    const unsigned long long launches0 = fmvd::rl_launch_count();
    ok = FMVD_CHECK(cudaStreamBeginCapture(origin, cudaStreamCaptureModeRelaxed)) &&
         FMVD_CHECK(cudaEventRecord(b->events[0], origin));
    for (int k = 0; k < nb && ok; k++)
        ok = FMVD_CHECK(cudaStreamWaitEvent(b->streams[1 + k], b->events[0], 0));
    for (int i = 0; i < count && ok; i++)
        ok = fmvd::engine_run(plans[i]->eng, d_views[i], view_strides[i], d_outs[i], nplanes[i], iterations[i],
                              nullptr, b->streams[1 + branch[i]]);
    for (int k = 0; k < nb && ok; k++)
        ok = FMVD_CHECK(cudaEventRecord(b->events[1 + k], b->streams[1 + k])) &&
             FMVD_CHECK(cudaStreamWaitEvent(origin, b->events[1 + k], 0));
    b->kernels = fmvd::rl_launch_count() - launches0;
    fmvd::rl_count_launch(0ull - b->kernels);  // captured, not launched
    cudaGraph_t graph = nullptr;
    const bool ended = FMVD_CHECK(cudaStreamEndCapture(origin, &graph));
    b->graph = graph;
    ok = ok && ended && graph && FMVD_CHECK(cudaGraphInstantiate(&b->exec, graph, 0));
    if (!ok) {
        release(b);
        return nullptr;
    }
    return b;
}

int fmvd_b200_batch_run(fmvd_b200_batch *batch, void *stream)
{
    if (!batch || !batch->exec) {
        fmvd::report_error("fmvd: invalid batch");
        return 1;
    }
    if (!FMVD_CHECK(cudaGraphLaunch(batch->exec, (cudaStream_t)stream)))
        return 1;
    fmvd::rl_count_launch(batch->kernels);
    return 0;
}

int fmvd_b200_batch_branches(const fmvd_b200_batch *batch) { return batch ? batch->branches : 0; }

void fmvd_b200_batch_destroy(fmvd_b200_batch *batch)
{
    if (!batch)
        return;
    cudaDeviceSynchronize();
    release(batch);
}

} // extern "C"
