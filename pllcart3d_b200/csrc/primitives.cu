// Stand-alone batched primitives of the reference's numerics on host
// buffers (used by the drop-in layer): pll_tridiag / tridiag_1rhs line
// solves, the 2-d DCT pair of fftw_3d.h, calculate_weno.  Default CUDA
// device and stream.
#include <cuda_runtime.h>

#include <vector>

#include "../../include/pllcart3d_gpu.h"
#include "dct_kernels.cuh"
#include "host_util.h"
#include "step_kernels.cuh"

using namespace pll;

namespace pll {
namespace {

// pll_tridiag's one-rank arithmetic on N contiguous systems of length n
__global__ void k_tridiag_batch(int N, int n, const double* __restrict__ a, double* __restrict__ b,
                                double* __restrict__ c, double* __restrict__ r)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const long o = (long)s * n;
    b[o] = b[o] - 0.0 * a[o];
    c[o] = c[o] / b[o];
    r[o] = (r[o] - 0.0 * a[o]) / b[o];
    for (int i = 1; i < n; ++i) {
        b[o + i] = (b[o + i] - c[o + i - 1] * a[o + i]);
        c[o + i] = c[o + i] / b[o + i];
        r[o + i] = (r[o + i] - r[o + i - 1] * a[o + i]) / b[o + i];
    }
    r[o + n - 1] = r[o + n - 1] - c[o + n - 1] * 0.0;
    for (int i = n - 2; i >= 0; --i) r[o + i] = r[o + i] - c[o + i] * r[o + i + 1];
}

}  // namespace
}  // namespace pll

extern "C" int pllgpu_tridiag_batch(int N, int n, const double* a, double* b, double* c, double* r)
{
    if (N < 0 || n < 1 || !a || !b || !c || !r) return PLLGPU_EINVAL;
    if (N == 0) return PLLGPU_OK;
    const size_t bytes = sizeof(double) * (size_t)N * n;
    DevBuf da, db, dc, dr;
    if (!da.alloc(bytes) || !db.alloc(bytes) || !dc.alloc(bytes) || !dr.alloc(bytes)) return PLLGPU_ECUDA;
    if (cudaMemcpy(da.p, a, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(db.p, b, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dc.p, c, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dr.p, r, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    k_tridiag_batch<<<(N + 127) / 128, 128>>>(N, n, da.d(), db.d(), dc.d(), dr.d());
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(b, db.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(c, dc.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(r, dr.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return PLLGPU_ECUDA;
    return PLLGPU_OK;
}

namespace pll {
namespace {

// the two contractions of a batched 2-d transform (along the fast
// dimension, then the slow one), in chunks of at most 65535 arrays (the
// grid's z limit)
void dct2d_gemms(int n0, int n1, int howmany, const double* x, const double* T0, const double* T1, double* tmp,
                 double* y)
{
    const long per = (long)n0 * n1;
    constexpr int kMaxZ = 65535;
    for (int b0 = 0; b0 < howmany; b0 += kMaxZ) {
        const int nb = (howmany - b0) < kMaxZ ? (howmany - b0) : kMaxZ;
        const long off = (long)b0 * per;
        const dim3 grid((n1 + 63) / 64, (n0 + 63) / 64, nb);
        // tmp[t][r][k] = sum_j T1[k][j] x[t][r][j]
        GemmDesc d1{n0, n1, n1, nb, per, n1, 1, 0, 1, n1, per, n1, 1, 0.0, 0};
        k_gemm_seq<double><<<grid, 256>>>(d1, x + off, T1, tmp + off);
        // y[t][k][c] = sum_r T0[k][r] tmp[t][r][c]
        GemmDesc d2{n0, n1, n0, nb, 0, n0, 1, per, n1, 1, per, n1, 1, 0.0, 0};
        k_gemm_seq<double><<<grid, 256>>>(d2, T0, tmp + off, y + off);
    }
}

}  // namespace
}  // namespace pll

extern "C" int pllgpu_dct2d_batch(int kind, int n0, int n1, int howmany, const double* in, double* out)
{
    if ((kind != 0 && kind != 1) || n0 < 1 || n1 < 1 || howmany < 0 || !in || !out) return PLLGPU_EINVAL;
    if (howmany == 0) return PLLGPU_OK;
    const long per = (long)n0 * n1;
    const size_t bytes = sizeof(double) * (size_t)per * howmany;
    std::vector<double> T0((size_t)n0 * n0), T1((size_t)n1 * n1);
    dct_matrix(kind, n0, T0.data());
    dct_matrix(kind, n1, T1.data());
    DevBuf dT0, dT1, dx, dtmp, dy;
    if (!dT0.alloc(sizeof(double) * T0.size()) || !dT1.alloc(sizeof(double) * T1.size()) || !dx.alloc(bytes) ||
        !dtmp.alloc(bytes) || !dy.alloc(bytes))
        return PLLGPU_ECUDA;
    if (cudaMemcpy(dT0.p, T0.data(), sizeof(double) * T0.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dT1.p, T1.data(), sizeof(double) * T1.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dx.p, in, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    dct2d_gemms(n0, n1, howmany, dx.d(), dT0.d(), dT1.d(), dtmp.d(), dy.d());
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(out, dy.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return PLLGPU_ECUDA;
    return PLLGPU_OK;
}


namespace pll {
namespace {

__global__ void k_weno_batch(int n, const double* __restrict__ v5, double* __restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double* v = v5 + 5L * t;
    out[t] = weno5<double>(v[0], v[1], v[2], v[3], v[4]);
}

// tridiag_1rhs on N contiguous systems; c' in scratch cc
__global__ void k_tridiag_1rhs_batch(int N, int n, const double* __restrict__ a, const double* __restrict__ b,
                                     const double* __restrict__ c, double* __restrict__ r, double* __restrict__ cc)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const long o = (long)s * n;
    double bb = b[o];
    cc[o] = c[o] / bb;
    r[o] = r[o] / bb;
    for (int i = 1; i < n; ++i) {
        bb = b[o + i] - cc[o + i - 1] * a[o + i];
        cc[o + i] = c[o + i] / bb;
        r[o + i] = (r[o + i] - r[o + i - 1] * a[o + i]) / bb;
    }
    for (int i = n - 2; i >= 0; --i) r[o + i] = r[o + i] - r[o + i + 1] * cc[o + i];
}

__global__ void k_divide(long n, double* __restrict__ x, double d)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) x[t] = x[t] / d;
}

}  // namespace
}  // namespace pll

extern "C" int pllgpu_weno_batch(int n, const double* v5, double* out)
{
    if (n < 0 || !v5 || !out) return PLLGPU_EINVAL;
    if (n == 0) return PLLGPU_OK;
    DevBuf dv, dout;
    if (!dv.alloc(sizeof(double) * 5 * (size_t)n) || !dout.alloc(sizeof(double) * (size_t)n)) return PLLGPU_ECUDA;
    if (cudaMemcpy(dv.p, v5, sizeof(double) * 5 * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    k_weno_batch<<<(n + 127) / 128, 128>>>(n, dv.d(), dout.d());
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(out, dout.p, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return PLLGPU_ECUDA;
    return PLLGPU_OK;
}

extern "C" int pllgpu_tridiag_1rhs_batch(int N, int n, const double* a, const double* b, const double* c,
                                         double* r)
{
    if (N < 0 || n < 1 || !a || !b || !c || !r) return PLLGPU_EINVAL;
    if (N == 0) return PLLGPU_OK;
    const size_t bytes = sizeof(double) * (size_t)N * n;
    DevBuf da, db, dc, dr, dcc;
    if (!da.alloc(bytes) || !db.alloc(bytes) || !dc.alloc(bytes) || !dr.alloc(bytes) || !dcc.alloc(bytes))
        return PLLGPU_ECUDA;
    if (cudaMemcpy(da.p, a, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(db.p, b, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dc.p, c, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dr.p, r, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    k_tridiag_1rhs_batch<<<(N + 127) / 128, 128>>>(N, n, da.d(), db.d(), dc.d(), dr.d(), dcc.d());
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(r, dr.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return PLLGPU_ECUDA;
    return PLLGPU_OK;
}

extern "C" int pllgpu_idct2d_batch(int n0, int n1, int howmany, const double* in, double* out)
{
    if (n0 < 1 || n1 < 1 || howmany < 0 || !in || !out) return PLLGPU_EINVAL;
    if (howmany == 0) return PLLGPU_OK;
    const long per = (long)n0 * n1, tot = per * howmany;
    const size_t bytes = sizeof(double) * (size_t)tot;
    std::vector<double> T0((size_t)n0 * n0), T1((size_t)n1 * n1);
    dct_matrix(1, n0, T0.data());
    dct_matrix(1, n1, T1.data());
    DevBuf dT0, dT1, dx, dtmp, dy;
    if (!dT0.alloc(sizeof(double) * T0.size()) || !dT1.alloc(sizeof(double) * T1.size()) || !dx.alloc(bytes) ||
        !dtmp.alloc(bytes) || !dy.alloc(bytes))
        return PLLGPU_ECUDA;
    if (cudaMemcpy(dT0.p, T0.data(), sizeof(double) * T0.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dT1.p, T1.data(), sizeof(double) * T1.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dx.p, in, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    dct2d_gemms(n0, n1, howmany, dx.d(), dT0.d(), dT1.d(), dtmp.d(), dy.d());
    // fftw_3d.h:101 divides by (double)(4*N)
    k_divide<<<(int)((tot + 255) / 256), 256>>>(tot, dy.d(), (double)(4 * per));
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(out, dy.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return PLLGPU_ECUDA;
    return PLLGPU_OK;
}
