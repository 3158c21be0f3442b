// Host-side helpers shared by the runtime and the two precision-form
// orchestration units (each translation unit keeps its own copy).
#pragma once

#include <cstdio>

#include "ctx.cuh"

namespace pll {
namespace {

int fail(pllgpu_ctx* c, int code)
{
    if (c && c->err == PLLGPU_OK) c->err = code;
    return code;
}

#define CK(call)                                                                     \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            std::fprintf(stderr, "pllgpu: %s failed: %s (%s:%d)\n", #call,           \
                         cudaGetErrorString(e_), __FILE__, __LINE__);                \
            return fail(ctx, PLLGPU_ECUDA);                                          \
        }                                                                            \
    } while (0)

// every kernel launch of the step: launched, or recorded while the context
// records (B: the kernel's batching spec, NoBatch where it has none)
template <typename B, typename... P, typename... A>
void go(pllgpu_ctx* ctx, void (*k)(P...), dim3 grid, dim3 blk, size_t smem, A&&... a)
{
    if (ctx->rec) {
        auto* r = new LaunchRecT<B, P...>();
        r->fn = (const void*)k;
        r->k = k;
        r->grid = grid;
        r->blk = blk;
        r->smem = smem;
        tup_fill(r->a, std::forward<A>(a)...);
        ctx->rec->push_back(r);
        return;
    }
    k<<<grid, blk, smem, ctx->st>>>(std::forward<A>(a)...);
}

// every kernel launch of the step goes through mark(): it counts launches
// and, in profiling mode, records an event after the launch so that the
// device time of each kernel is the gap to the previous event
void mark(pllgpu_ctx* ctx, const char* label)
{
    ctx->counting++;
    if (!ctx->profiling) return;
    const size_t i = ctx->ev_label.size();
    if (i >= ctx->ev_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ctx->ev_pool.push_back(e);
    }
    cudaEventRecord(ctx->ev_pool[i], ctx->st);
    ctx->ev_label.push_back(label);
}

template <typename T>
T* dalloc(pllgpu_ctx* ctx, long n)
{
    void* p = nullptr;
    // 1 KB of zeroed slack past the end: kernels that compute cell pairs
    // (k_explicit2) read, and never write, up to 66 elements beyond a field
    const size_t bytes = sizeof(T) * (size_t)(n > 0 ? n : 1) + 1024;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, bytes);
    ctx->allocs.push_back(p);
    return (T*)p;
}

dim3 box_grid(int nk, int nj, int ni, dim3 blk)
{
    return dim3((nk + blk.x - 1) / blk.x, (nj + blk.y - 1) / blk.y, ni);
}

int ni(const Rng& r) { return r.ie - r.is + 1; }
int nj(const Rng& r) { return r.je - r.js + 1; }
int nk(const Rng& r) { return r.ke - r.ks + 1; }

int set_scalar(pllgpu_ctx* ctx, int slot, double v)
{
    CK(cudaMemcpyAsync(ctx->scal + slot, &v, sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

double get_scalar(pllgpu_ctx* ctx, int slot)
{
    double v = NAN;
    if (cudaMemcpyAsync(&v, ctx->scal + slot, sizeof(double), cudaMemcpyDeviceToHost, ctx->st) != cudaSuccess ||
        cudaStreamSynchronize(ctx->st) != cudaSuccess)
        fail(ctx, PLLGPU_ECUDA);
    return v;
}

int check_launch(pllgpu_ctx* ctx)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "pllgpu: kernel launch failed: %s\n", cudaGetErrorString(e));
        return fail(ctx, PLLGPU_ECUDA);
    }
    return PLLGPU_OK;
}

int read_status(pllgpu_ctx* ctx)
{
    int s = 0;
    CK(cudaMemcpyAsync(&s, ctx->status, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (s & ST_NAN) return fail(ctx, PLLGPU_ENAN);
    if (s & ST_NOCONV) return fail(ctx, PLLGPU_ENOCONV);
    if (s & ST_BOUNDS) return fail(ctx, PLLGPU_EBOUNDS);
    if (s & ST_TIMEOUT) return fail(ctx, PLLGPU_ETIMEOUT);
    return PLLGPU_OK;
}

__global__ void k_convert_to_f32(long n, const double* __restrict__ a, float* __restrict__ b)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = (float)a[t];
}

__global__ void k_convert_to_f64(long n, const float* __restrict__ a, double* __restrict__ b)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = (double)a[t];
}

}  // namespace
}  // namespace pll
