// Ensembles of independent runs (grids and parameters may all differ)
// advanced together: every member is an ordinary context with its own
// stream and state in HBM; one CUDA graph holds one full step of every member
// as parallel branches (fork from a root stream, each member's kernels on its
// own stream, join back), so a single graph launch advances the whole
// ensemble and the kernels of different members share the SMs.  Small grids
// that leave most of the GPU idle on their own fill it together.
//
// Each member computes exactly what it computes alone (the same kernels with
// the same arithmetic on its own buffers); the autotuner picks each member's
// launch shapes from variants that are bit-identical by construction.
#include <cuda_runtime.h>

#include <vector>

#include "../../include/pllcart3d_gpu.h"
#include "forms.h"
#include "host_common.cuh"

using namespace pll;

struct pllgpu_ensemble {
    std::vector<pllgpu_ctx*> m;
    int dev = 0;
    cudaStream_t root = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    bool ready = false;
    int launches_per_step = 0;
};

namespace {

void drop_graphs(pllgpu_ensemble* e)
{
    for (int t = 0; t < 2; ++t)
        if (e->gexec[t]) {
            cudaGraphExecDestroy(e->gexec[t]);
            e->gexec[t] = nullptr;
        }
    e->ready = false;
}

// one step of every member enqueued on its own stream, forked from and
// joined back into the root stream
int enqueue_all(pllgpu_ensemble* e)
{
    if (cudaEventRecord(e->fork, e->root) != cudaSuccess) return PLLGPU_ECUDA;
    int launches = 0;
    for (size_t i = 0; i < e->m.size(); ++i) {
        pllgpu_ctx* c = e->m[i];
        if (cudaStreamWaitEvent(c->st, e->fork, 0) != cudaSuccess) return PLLGPU_ECUDA;
        c->counting = 0;
        enqueue_step_any(c);
        launches += c->counting;
        if (cudaEventRecord(e->join[i], c->st) != cudaSuccess) return PLLGPU_ECUDA;
        if (cudaStreamWaitEvent(e->root, e->join[i], 0) != cudaSuccess) return PLLGPU_ECUDA;
    }
    e->launches_per_step = launches;
    return PLLGPU_OK;
}

int build(pllgpu_ensemble* e)
{
    for (int t = 0; t < 2; ++t) {
        const int parity = e->m[0]->cur;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(e->root, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return PLLGPU_ECUDA;
        const int rc = enqueue_all(e);
        if (cudaStreamEndCapture(e->root, &g) != cudaSuccess || rc) {
            if (g) cudaGraphDestroy(g);
            return PLLGPU_ECUDA;
        }
        const cudaError_t ie = cudaGraphInstantiate(&e->gexec[parity], g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return PLLGPU_ECUDA;
        // every member's cur flipped once during the capture
    }
    e->ready = true;
    return PLLGPU_OK;
}

int members_status(pllgpu_ensemble* e)
{
    int first = PLLGPU_OK;
    for (pllgpu_ctx* c : e->m) {
        const int s = read_status(c);
        if (s && !first) first = s;
    }
    return first;
}

}  // namespace

extern "C" {

pllgpu_ensemble* pllgpu_ensemble_create(int n, const pllgpu_params* params, int device)
{
    if (n < 1 || !params) return nullptr;
    pllgpu_ensemble* e = new pllgpu_ensemble();
    e->dev = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&e->root, cudaStreamNonBlocking) ||
        cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming)) {
        delete e;
        return nullptr;
    }
    for (int i = 0; i < n; ++i) {
        pllgpu_ctx* c = pllgpu_create(&params[i], device);
        cudaEvent_t j = nullptr;
        if (!c || cudaEventCreateWithFlags(&j, cudaEventDisableTiming) != cudaSuccess) {
            if (c) pllgpu_destroy(c);
            pllgpu_ensemble_destroy(e);
            return nullptr;
        }
        e->m.push_back(c);
        e->join.push_back(j);
    }
    return e;
}

void pllgpu_ensemble_destroy(pllgpu_ensemble* e)
{
    if (!e) return;
    cudaSetDevice(e->dev);
    if (e->root) cudaStreamSynchronize(e->root);
    drop_graphs(e);
    for (pllgpu_ctx* c : e->m) pllgpu_destroy(c);
    for (cudaEvent_t j : e->join) cudaEventDestroy(j);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->root) cudaStreamDestroy(e->root);
    delete e;
}

int pllgpu_ensemble_size(const pllgpu_ensemble* e) { return e ? (int)e->m.size() : 0; }

pllgpu_ctx* pllgpu_ensemble_member(pllgpu_ensemble* e, int i)
{
    if (!e || i < 0 || i >= (int)e->m.size()) return nullptr;
    return e->m[i];
}

int pllgpu_ensemble_start(pllgpu_ensemble* e)
{
    if (!e) return PLLGPU_EINVAL;
    for (pllgpu_ctx* c : e->m)
        if (int s = pllgpu_start(c)) return s;
    drop_graphs(e);
    return PLLGPU_OK;
}

int pllgpu_ensemble_steps(pllgpu_ensemble* e, int nsteps)
{
    if (!e || nsteps < 0) return PLLGPU_EINVAL;
    if (cudaSetDevice(e->dev) != cudaSuccess) return PLLGPU_ECUDA;
    if (nsteps == 0) return PLLGPU_OK;
    // all members must share the buffer parity (they start and step
    // together); a member restarted from files takes its first step on the
    // streams (it carries the restart copy)
    bool stream_step = false;
    for (pllgpu_ctx* c : e->m) {
        if (c->cur != e->m[0]->cur) return PLLGPU_EINVAL;   // members stepped apart
        stream_step |= c->resync_c;
    }
    if (stream_step) {
        if (enqueue_all(e)) return PLLGPU_ECUDA;
        --nsteps;
        drop_graphs(e);
    }
    if (!e->ready) {
        if (int s = build(e)) return s;
    }
    for (int s = 0; s < nsteps; ++s) {
        const int parity = e->m[0]->cur;
        if (cudaGraphLaunch(e->gexec[parity], e->root) != cudaSuccess) return PLLGPU_ECUDA;
        for (pllgpu_ctx* c : e->m) c->cur ^= 1;
    }
    if (cudaStreamSynchronize(e->root) != cudaSuccess) return PLLGPU_ECUDA;
    for (pllgpu_ctx* c : e->m) c->rotated = true;
    return members_status(e);
}

int pllgpu_ensemble_autotune(pllgpu_ensemble* e, int trial_steps, int* steps_done)
{
    if (!e) return PLLGPU_EINVAL;
    int done = -1;
    for (pllgpu_ctx* c : e->m) {
        int d = 0;
        if (int s = pllgpu_autotune(c, trial_steps, &d)) return s;
        if (done >= 0 && d != done) return PLLGPU_EINVAL;   // parities would diverge
        done = d;
    }
    drop_graphs(e);
    if (steps_done) *steps_done = done;
    return PLLGPU_OK;
}

int pllgpu_ensemble_launches_per_step(const pllgpu_ensemble* e) { return e ? e->launches_per_step : 0; }

}  // extern "C"
