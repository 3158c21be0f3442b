// Batched 2-d DCT (the transform pair of phisolver_dct) that allocates no
// device memory.
//
// pllgpu_dct2d_batch allocates device buffers on every call (cudaMalloc /
// cudaFree), which not every caller can afford: a host that hands all of
// its device memory to its own pool allocator has nothing left for
// out-of-band allocations, and cudaMalloc/cudaFree may synchronize the
// device, which a caller streaming work on its own stream cannot accept.
// pllgpu_dct2d_batch_noalloc takes the caller's device buffers for input and
// output and keeps its two cosine matrices and its intermediate array in a
// fixed scratch array that belongs to the library, so a call allocates
// nothing.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "../../include/pllcart3d_gpu.h"
#include "dct_kernels.cuh"

using namespace pll;

// Scratch of the no-allocation DCT: 2^21 doubles (16 MiB).  Every GPU that
// loads the library holds one copy until the process exits.  All calls share
// it and it keeps the previous call's contents; every call overwrites the
// part it reads before reading it, so nothing needs clearing.
static __device__ __align__(256) double g_dct_scratch[PLLGPU_DCT_NOALLOC_MAX_DOUBLES];

namespace pll {
namespace {

constexpr int kMaxDevices = 64;
// device address of g_dct_scratch per device (the host-side symbol is only a
// stand-in and must never be handed to a kernel)
double* g_scratch_addr[kMaxDevices] = {};

// FFTW REDFT10 / REDFT01 matrices T[k*n+j] written on the device, with the
// argument reduced mod 4n exactly as on the host side
__global__ void k_dct_matrix(int kind, int n, double* T)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * n) return;
    const int k = (int)(t / n), j = (int)(t % n);
    const double pi = 3.14159265358979323846;
    double v;
    if (kind == 0) {
        const long m = ((long)(2 * j + 1) * (long)k) % (4L * n);
        v = 2.0 * cos(pi * (double)m / (2.0 * n));
    } else if (j == 0) {
        v = 1.0;
    } else {
        const long m = ((long)j * (long)(2 * k + 1)) % (4L * n);
        v = 2.0 * cos(pi * (double)m / (2.0 * n));
    }
    T[t] = v;
}

}  // namespace
}  // namespace pll

namespace pll {
namespace {

// Scratch doubles a call needs (n0*n0 + n1*n1 + howmany*n0*n1), or -1 when
// that exceeds the fixed array.  Each term is bounded before it is added,
// so no product or sum can overflow (n0, n1, howmany >= 1).
long noalloc_need(int n0, int n1, int howmany)
{
    const long cap = (long)PLLGPU_DCT_NOALLOC_MAX_DOUBLES;
    const long t0 = (long)n0 * n0, t1 = (long)n1 * n1, per = (long)n0 * n1;   // < 2^62 each
    if (t0 > cap || t1 > cap || per > cap || t0 + t1 > cap) return -1;
    if ((long)howmany > (cap - t0 - t1) / per) return -1;
    return t0 + t1 + per * howmany;
}

// one launch with its own error code (cudaLaunchKernel returns the error of
// this launch; the thread's pending error is touched only when it failed)
cudaError_t launch(const void* fn, dim3 grid, dim3 block, void** args, cudaStream_t st)
{
    const cudaError_t e = cudaLaunchKernel(fn, grid, block, args, 0, st);
    if (e != cudaSuccess) (void)cudaGetLastError();   // the error is this launch's; report it by return
    return e;
}

}  // namespace
}  // namespace pll

extern "C" int pllgpu_dct2d_batch_noalloc(int kind, int n0, int n1, int howmany, const double* d_in,
                                          double* d_out, void* stream)
{
    if ((kind != 0 && kind != 1) || n0 < 1 || n1 < 1 || howmany < 0 || !d_in || !d_out) return PLLGPU_EINVAL;
    if (howmany == 0) return PLLGPU_OK;
    if (noalloc_need(n0, n1, howmany) < 0) {
        std::fprintf(stderr,
                     "pllgpu_dct2d_batch_noalloc: %d x %d x %d needs more than its fixed scratch of %ld "
                     "doubles\n",
                     howmany, n0, n1, (long)PLLGPU_DCT_NOALLOC_MAX_DOUBLES);
        return PLLGPU_EINVAL;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PLLGPU_ECUDA;
    if (!g_scratch_addr[dev]) {
        // one-time set-up on this device (with it current): the device
        // address of the scratch array
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_dct_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "pllgpu_dct2d_batch_noalloc: cudaGetSymbolAddress failed: %s\n",
                         cudaGetErrorString(e));
            return PLLGPU_ECUDA;
        }
        g_scratch_addr[dev] = (double*)p;
    }
    cudaStream_t st = (cudaStream_t)stream;
    double* T0 = g_scratch_addr[dev];
    double* T1 = T0 + (long)n0 * n0;
    double* tmp = T1 + (long)n1 * n1;
    const long per = (long)n0 * n1;
    {
        int kd = kind, n = n0;
        double* T = T0;
        void* args[] = {&kd, &n, &T};
        if (launch((const void*)k_dct_matrix, dim3((unsigned)(((long)n0 * n0 + 255) / 256)), dim3(256), args, st) !=
            cudaSuccess)
            return PLLGPU_ECUDA;
        n = n1;
        T = T1;
        if (launch((const void*)k_dct_matrix, dim3((unsigned)(((long)n1 * n1 + 255) / 256)), dim3(256), args, st) !=
            cudaSuccess)
            return PLLGPU_ECUDA;
    }
    // along the fast dimension, then along the slow one (as
    // pllgpu_dct2d_batch); the batch goes in chunks that fit gridDim.z
    constexpr int kMaxZ = 65535;
    for (int b0 = 0; b0 < howmany; b0 += kMaxZ) {
        const int nb = (howmany - b0) < kMaxZ ? (howmany - b0) : kMaxZ;
        const double* in = d_in + (long)b0 * per;
        double* t = tmp + (long)b0 * per;
        double* out = d_out + (long)b0 * per;
        const dim3 grid((unsigned)((n1 + 63) / 64), (unsigned)((n0 + 63) / 64), (unsigned)nb);
        GemmDesc a{n0, n1, n1, nb, per, n1, 1, 0, 1, n1, per, n1, 1, 0.0, 0};
        const double* B1 = T1;
        void* args_a[] = {&a, &in, &B1, &t};
        if (launch((const void*)k_gemm_seq<double>, grid, dim3(256), args_a, st) != cudaSuccess) return PLLGPU_ECUDA;
        GemmDesc b{n0, n1, n0, nb, 0, n0, 1, per, n1, 1, per, n1, 1, 0.0, 0};
        const double* A0 = T0;
        const double* tc = t;
        void* args_b[] = {&b, &A0, &tc, &out};
        if (launch((const void*)k_gemm_seq<double>, grid, dim3(256), args_b, st) != cudaSuccess) return PLLGPU_ECUDA;
    }
    return PLLGPU_OK;
}
