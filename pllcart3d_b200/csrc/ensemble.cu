// Ensembles of independent runs (grids and parameters may all differ)
// advanced together: every member is an ordinary context with its own state
// in HBM, and one CUDA graph launch advances the whole ensemble one step.
//
// Members whose steps issue the same launches (same kernels, shapes and
// shared memory: in practice the same grid and form) form a class.  The
// graph holds one branch per class, and in it one launch per stage for the
// whole class: the stage's kernel body runs over a grid whose z extent is
// the class size times the member's, each member reading its own arguments
// from a device table (batch.cuh).  64 members on 4 grid classes so issue 4
// launches per stage, not 64.  Stages whose kernels take a tensor map
// (none in the precision form at these grid sizes) issue one launch per
// member in the class's branch.
//
// Each member computes exactly what it computes alone (the same kernel body
// with the same arithmetic on its own buffers); the autotuner picks launch
// shapes from variants that are bit-identical by construction, and gives
// every member of a grid the same ones so that they batch.
#include <cuda_runtime.h>

#include <cstring>
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
    bool batching = true;
    int group = 0;                     // members per batched launch at most (0: whole classes)
    int launches_per_step = 0;
    int classes = 0;
    unsigned char* tables = nullptr;   // device argument tables of the batched launches
};

namespace {

void drop_graphs(pllgpu_ensemble* e)
{
    for (int t = 0; t < 2; ++t)
        if (e->gexec[t]) {
            cudaGraphExecDestroy(e->gexec[t]);
            e->gexec[t] = nullptr;
        }
    if (e->tables) {
        cudaFree(e->tables);
        e->tables = nullptr;
    }
    e->ready = false;
    e->classes = 0;
}

typedef std::vector<LaunchRec*> Recs;

void free_recs(std::vector<Recs>& r)
{
    for (Recs& v : r)
        for (LaunchRec* x : v) delete x;
    r.clear();
}

// one step of member c recorded instead of issued.  The recording runs
// inside a capture of the member's stream that is then thrown away: a launch
// that bypassed the recorder would land in that graph, not on the GPU, and
// is detected by its node count.
bool record_step(pllgpu_ctx* c, Recs& out)
{
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
    c->rec = &out;
    c->counting = 0;
    enqueue_step_any(c);
    c->rec = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->st, &g);
    size_t nodes = 1;
    if (ec == cudaSuccess && g) cudaGraphGetNodes(g, nullptr, &nodes);
    if (g) cudaGraphDestroy(g);
    return ec == cudaSuccess && nodes == 0 && c->err == PLLGPU_OK;
}

bool same_steps(const Recs& a, const Recs& b)
{
    if (a.size() != b.size()) return false;
    for (size_t p = 0; p < a.size(); ++p)
        if (!a[p]->same_launch(*b[p])) return false;
    return true;
}

size_t pack_stride(const LaunchRec* r) { return (r->arg_bytes() + 127) / 128 * 128; }

// the batched graphs: both parities' steps of every member recorded, the
// members split into classes of identical steps, every class's argument
// tables in one device allocation, then one capture per parity with one
// branch per class
int build_batched(pllgpu_ensemble* e)
{
    const size_t n = e->m.size();
    std::vector<Recs> rec[2];
    int parity[2];
    for (int t = 0; t < 2; ++t) {
        parity[t] = e->m[0]->cur;
        rec[t].resize(n);
        for (size_t i = 0; i < n; ++i)
            if (!record_step(e->m[i], rec[t][i])) {
                std::fprintf(stderr, "pllgpu: ensemble: recording member %zu's step failed\n", i);
                // every recorded step flipped its member's parity: undo
                for (pllgpu_ctx* c : e->m) c->cur = parity[0];
                free_recs(rec[0]);
                free_recs(rec[1]);
                return PLLGPU_ECUDA;
            }
    }
    // classes: members whose two recorded steps match launch for launch
    std::vector<std::vector<int>> cls;
    for (size_t i = 0; i < n; ++i) {
        bool placed = false;
        for (auto& c : cls)
            if (same_steps(rec[0][c[0]], rec[0][i]) && same_steps(rec[1][c[0]], rec[1][i])) {
                c.push_back((int)i);
                placed = true;
                break;
            }
        if (!placed) cls.push_back({(int)i});
    }
    // classes above the group limit split into groups of at most that many
    // members, each its own branch (more branches overlap one another's
    // kernel tails; fewer launches per step the larger the groups)
    if (e->group > 1) {
        std::vector<std::vector<int>> split;
        for (auto& c : cls)
            for (size_t k0 = 0; k0 < c.size(); k0 += (size_t)e->group)
                split.emplace_back(c.begin() + k0, c.begin() + std::min(c.size(), k0 + (size_t)e->group));
        cls.swap(split);
    }
    // argument tables: per parity, class and batched launch, the members'
    // packs at a 128-byte stride
    std::vector<size_t> off[2];
    size_t total = 0;
    for (int t = 0; t < 2; ++t)
        for (auto& c : cls) {
            if (c.size() < 2) continue;
            for (const LaunchRec* r : rec[t][c[0]]) {
                off[t].push_back(total);
                if (r->batchable()) total += pack_stride(r) * c.size();
            }
        }
    std::vector<unsigned char> host(total ? total : 1, 0);
    for (int t = 0; t < 2; ++t) {
        size_t q = 0;
        for (auto& c : cls) {
            if (c.size() < 2) continue;
            for (size_t p = 0; p < rec[t][c[0]].size(); ++p, ++q) {
                const LaunchRec* r = rec[t][c[0]][p];
                if (!r->batchable()) continue;
                for (size_t k = 0; k < c.size(); ++k)
                    std::memcpy(host.data() + off[t][q] + k * pack_stride(r), rec[t][c[k]][p]->arg_data(),
                                r->arg_bytes());
            }
        }
    }
    int rc = PLLGPU_OK;
    auto bad = [&](const char* what, cudaError_t err) {
        std::fprintf(stderr, "pllgpu: ensemble: %s: %s\n", what, cudaGetErrorString(err));
        rc = PLLGPU_ECUDA;
    };
    if (total) {
        cudaError_t err = cudaMalloc(&e->tables, total);
        if (err == cudaSuccess) err = cudaMemcpy(e->tables, host.data(), total, cudaMemcpyHostToDevice);
        if (err != cudaSuccess) bad("argument tables", err);
    }
    for (int t = 0; t < 2 && rc == PLLGPU_OK; ++t)
        for (auto& c : cls)
            for (const LaunchRec* r : rec[t][c[0]])
                if (c.size() >= 2 && r->batchable() && rc == PLLGPU_OK)
                    if (cudaError_t err = r->prepare()) bad("shared-memory opt-in", err);
    int launches = 0;
    for (int t = 0; t < 2 && rc == PLLGPU_OK; ++t) {
        cudaGraph_t g = nullptr;
        if (cudaError_t err = cudaStreamBeginCapture(e->root, cudaStreamCaptureModeThreadLocal)) {
            bad("capture", err);
            break;
        }
        bool ok = cudaEventRecord(e->fork, e->root) == cudaSuccess;
        launches = 0;
        size_t q = 0;
        for (size_t ci = 0; ci < cls.size() && ok; ++ci) {
            const auto& c = cls[ci];
            cudaStream_t st = e->m[c[0]]->st;
            ok = cudaStreamWaitEvent(st, e->fork, 0) == cudaSuccess;
            for (size_t p = 0; p < rec[t][c[0]].size() && ok; ++p) {
                const LaunchRec* r = rec[t][c[0]][p];
                if (c.size() < 2 || !r->batchable()) {
                    for (int k : c) rec[t][k][p]->one(st);
                    launches += (int)c.size();
                } else {
                    // grid.z of one launch stays within 65535: chunks of members
                    const size_t stride = pack_stride(r);
                    const size_t chunk = std::max<size_t>(1, 65535 / std::max(1u, r->grid.z));
                    for (size_t k0 = 0; k0 < c.size() && ok; k0 += chunk) {
                        const unsigned cn = (unsigned)std::min(chunk, c.size() - k0);
                        if (cudaError_t err = r->many(e->tables + off[t][q] + k0 * stride, stride, cn, st)) {
                            std::fprintf(stderr,
                                         "pllgpu: ensemble: batched launch %zu (grid %u %u %u x %u, block %u %u %u, "
                                         "%zu bytes shared): %s\n", p, r->grid.x, r->grid.y, r->grid.z, cn,
                                         r->blk.x, r->blk.y, r->blk.z, r->smem, cudaGetErrorString(err));
                            ok = false;
                        }
                        ++launches;
                    }
                }
                if (c.size() >= 2) ++q;
            }
            if (ok) ok = cudaEventRecord(e->join[ci], st) == cudaSuccess &&
                         cudaStreamWaitEvent(e->root, e->join[ci], 0) == cudaSuccess;
        }
        const cudaError_t ee = cudaStreamEndCapture(e->root, &g);
        if (!ok || ee != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            bad("capture", ee != cudaSuccess ? ee : cudaErrorInvalidValue);
            break;
        }
        const cudaError_t ie = cudaGraphInstantiate(&e->gexec[parity[t]], g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) bad("graph instantiation", ie);
    }
    free_recs(rec[0]);
    free_recs(rec[1]);
    if (rc != PLLGPU_OK) {
        drop_graphs(e);
        return rc;
    }
    // the two recordings flipped every member's parity twice: back where it was
    e->launches_per_step = launches;
    e->classes = (int)cls.size();
    e->ready = true;
    return PLLGPU_OK;
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

// one branch per member, each member's own launches (no batching)
int build_branches(pllgpu_ensemble* e)
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
    e->classes = (int)e->m.size();
    e->ready = true;
    return PLLGPU_OK;
}

int build(pllgpu_ensemble* e) { return e->batching ? build_batched(e) : build_branches(e); }

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
    // members of one grid and form take the first one's variants (all
    // variants give the same bits), so that their launches batch
    for (size_t i = 1; i < e->m.size(); ++i)
        for (size_t j = 0; j < i; ++j) {
            const pllgpu_ctx *a = e->m[j], *b = e->m[i];
            if (a->mixed == b->mixed && a->P.precision == b->P.precision && a->G.nx == b->G.nx &&
                a->G.ny == b->G.ny && a->G.nz == b->G.nz) {
                if (int s = pllgpu_set_tuning(e->m[i], a->tune_exp, a->tune_line)) return s;
                break;
            }
        }
    drop_graphs(e);
    if (steps_done) *steps_done = done;
    return PLLGPU_OK;
}

int pllgpu_ensemble_launches_per_step(const pllgpu_ensemble* e) { return e ? e->launches_per_step : 0; }

int pllgpu_ensemble_set_batching(pllgpu_ensemble* e, int mode)
{
    if (!e || mode < 0) return -PLLGPU_EINVAL;
    const int old = !e->batching ? 0 : e->group > 1 ? e->group : 1;
    if (mode != old) {
        e->batching = mode != 0;
        e->group = mode > 1 ? mode : 0;
        drop_graphs(e);
    }
    return old;
}

int pllgpu_ensemble_classes(const pllgpu_ensemble* e) { return e ? e->classes : 0; }

}  // extern "C"
