// Batched dense contractions for the DCT-II / DCT-III of the Poisson solve
// (phisolver_dct pllcart3d.c:2035, 2104 through fftw_3d.h:45-106).  Each
// 1-d transform is a product with a dense cosine matrix (FFTW's documented
// REDFT10/REDFT01 definitions); the 2-d transform of an x-plane is the y
// pass followed by the z pass.
#pragma once

#include <cuda_runtime.h>

namespace pll {

struct GemmDesc {
    int M, N, K, batch;
    long sAb, sAm, sAk;
    long sBb, sBk, sBn;
    long sCb, sCm, sCn;
    double scale;   // output multiplier (scale_mode 1) or divisor (mode 2)
    int scale_mode;
};

// C[b][m][n] = sum_k A[b][m][k] * B[b][k][n], accumulated in increasing k,
// acc = acc + a*b, from 0 (the summation order of a sequential loop).
// 64x64 output tile per 256-thread block, 4x4 outputs per thread.
template <typename real>
__global__ void __launch_bounds__(256) k_gemm_seq(GemmDesc d, const real* __restrict__ A,
                                                  const real* __restrict__ B, real* __restrict__ C)
{
    constexpr int TM = 64, TN = 64, TK = 16;
    __shared__ real As[TK][TM + 1];
    __shared__ real Bs[TK][TN + 1];
    const int b = blockIdx.z;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const real* Ab = A + (long)b * d.sAb;
    const real* Bb = B + (long)b * d.sBb;
    real acc[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = (real)0;
    for (int k0 = 0; k0 < d.K; k0 += TK) {
        // consecutive threads walk the operand's unit-stride index
        for (int t = threadIdx.x; t < TK * TM; t += 256) {
            const int kk = d.sAk == 1 ? t % TK : t / TM, mm = d.sAk == 1 ? t / TK : t % TM;
            const int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < d.M && k < d.K) ? Ab[(long)m * d.sAm + (long)k * d.sAk] : (real)0;
        }
        for (int t = threadIdx.x; t < TK * TN; t += 256) {
            const int kk = d.sBk == 1 ? t % TK : t / TN, nn = d.sBk == 1 ? t / TK : t % TN;
            const int n = n0 + nn, k = k0 + kk;
            Bs[kk][nn] = (n < d.N && k < d.K) ? Bb[(long)k * d.sBk + (long)n * d.sBn] : (real)0;
        }
        __syncthreads();
        const int kmax = (d.K - k0) < TK ? (d.K - k0) : TK;
        for (int kk = 0; kk < kmax; ++kk) {
            real a[4], bv[4];
#pragma unroll
            for (int p = 0; p < 4; ++p) a[p] = As[kk][ty + 16 * p];
#pragma unroll
            for (int q = 0; q < 4; ++q) bv[q] = Bs[kk][tx + 16 * q];
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[p][q] = acc[p][q] + a[p] * bv[q];
        }
        __syncthreads();
    }
    real* Cb = C + (long)b * d.sCb;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int m = m0 + ty + 16 * p;
        if (m >= d.M) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int n = n0 + tx + 16 * q;
            if (n >= d.N) continue;
            real v = acc[p][q];
            if (d.scale_mode == 1) v = v * (real)d.scale;
            else if (d.scale_mode == 2) v = v / (real)d.scale;
            Cb[(long)m * d.sCm + (long)n * d.sCn] = v;
        }
    }
}

}  // namespace pll
