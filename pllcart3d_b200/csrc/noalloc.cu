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

extern "C" int pllgpu_dct2d_batch_noalloc(int kind, int n0, int n1, int howmany, const double* d_in,
                                          double* d_out, void* stream)
{
    if ((kind != 0 && kind != 1) || n0 < 1 || n1 < 1 || howmany < 0 || !d_in || !d_out) return PLLGPU_EINVAL;
    if (howmany == 0) return PLLGPU_OK;
    const long per = (long)n0 * n1;
    const long need = (long)n0 * n0 + (long)n1 * n1 + per * howmany;
    if (need > (long)PLLGPU_DCT_NOALLOC_MAX_DOUBLES) {
        std::fprintf(stderr,
                     "pllgpu_dct2d_batch_noalloc: %d x %d x %d needs %ld doubles of scratch, "
                     "more than its fixed %ld\n",
                     howmany, n0, n1, need, (long)PLLGPU_DCT_NOALLOC_MAX_DOUBLES);
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
    k_dct_matrix<<<(int)(((long)n0 * n0 + 255) / 256), 256, 0, st>>>(kind, n0, T0);
    k_dct_matrix<<<(int)(((long)n1 * n1 + 255) / 256), 256, 0, st>>>(kind, n1, T1);
    // along the fast dimension, then along the slow one (as pllgpu_dct2d_batch)
    GemmDesc a{n0, n1, n1, howmany, per, n1, 1, 0, 1, n1, per, n1, 1, 0.0, 0};
    k_gemm_seq<double><<<dim3((n1 + 63) / 64, (n0 + 63) / 64, howmany), 256, 0, st>>>(a, d_in, T1, tmp);
    GemmDesc b{n0, n1, n0, howmany, 0, n0, 1, per, n1, 1, per, n1, 1, 0.0, 0};
    k_gemm_seq<double><<<dim3((n1 + 63) / 64, (n0 + 63) / 64, howmany), 256, 0, st>>>(b, T0, tmp, d_out);
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    return PLLGPU_OK;
}
