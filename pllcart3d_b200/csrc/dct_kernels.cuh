// Batched dense contractions for the DCT-II / DCT-III of the Poisson solve
// (phisolver_dct pllcart3d.c:2035, 2104 through fftw_3d.h:45-106).  Each
// 1-d transform is a product with a dense cosine matrix (FFTW's documented
// REDFT10/REDFT01 definitions); the 2-d transform of an x-plane is the y
// pass followed by the z pass.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace pll {
// internal linkage: each translation unit (and so each precision form with
// its own contraction flags) owns its instantiations
namespace {

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
__device__ __forceinline__ void k_gemm_seq_run(const uint3 blockIdx, const dim3 gridDim,
    GemmDesc d, const real* __restrict__ A,
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
template <typename real>
__global__ void __launch_bounds__(256) k_gemm_seq(GemmDesc d, const real* __restrict__ A,
                                                  const real* __restrict__ B, real* __restrict__ C)
{
    k_gemm_seq_run<real>(blockIdx, gridDim, d, A, B, C);
}
template <typename real>
struct k_gemm_seq_b {
    static constexpr auto run = &k_gemm_seq_run<real>;
    static constexpr int maxt = 256, minb = 0;
};


// Same contraction on the FP64 tensor cores: mma.sync m8n8k4 .f64 (DMMA),
// FP64 products and FP64 accumulation in the tensor pipe (the order of the
// k-sum differs from the sequential loop, so results agree with k_gemm_seq
// to rounding).  64x64 block tile, 8 warps as 2 (m) x 4 (n), each warp a
// 32x16 sub-tile of 4x2 m8n8 fragments; k tiles of 16 through shared memory.
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

static __device__ __forceinline__ void k_gemm_dmma_run(const uint3 blockIdx, const dim3 gridDim,
    GemmDesc d, const double* __restrict__ A,
                                                   const double* __restrict__ B, double* __restrict__ C)
{
    constexpr int TM = 64, TN = 64, TK = 16, PAD = 4;
    __shared__ double As[TK][TM + PAD];
    __shared__ double Bs[TK][TN + PAD];
    const int b = blockIdx.z;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp >> 2, wn = warp & 3;   // 2 x 4 warps
    const int g = lane >> 2, tg = lane & 3;    // fragment group / thread in group
    const double* Ab = A + (long)b * d.sAb;
    const double* Bb = B + (long)b * d.sBb;
    double acc[4][2][2];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 2; ++q) acc[p][q][0] = acc[p][q][1] = 0.0;
    for (int k0 = 0; k0 < d.K; k0 += TK) {
        for (int t = threadIdx.x; t < TK * TM; t += 256) {
            const int kk = d.sAk == 1 ? t % TK : t / TM, mm = d.sAk == 1 ? t / TK : t % TM;
            const int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < d.M && k < d.K) ? Ab[(long)m * d.sAm + (long)k * d.sAk] : 0.0;
        }
        for (int t = threadIdx.x; t < TK * TN; t += 256) {
            const int kk = d.sBk == 1 ? t % TK : t / TN, nn = d.sBk == 1 ? t / TK : t % TN;
            const int n = n0 + nn, k = k0 + kk;
            Bs[kk][nn] = (n < d.N && k < d.K) ? Bb[(long)k * d.sBk + (long)n * d.sBn] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; kk += 4) {
            double a[4], bv[2];
#pragma unroll
            for (int p = 0; p < 4; ++p) a[p] = As[kk + tg][wm * 32 + p * 8 + g];
#pragma unroll
            for (int q = 0; q < 2; ++q) bv[q] = Bs[kk + tg][wn * 16 + q * 8 + g];
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 2; ++q) dmma_8x8x4(acc[p][q][0], acc[p][q][1], a[p], bv[q]);
        }
        __syncthreads();
    }
    double* Cb = C + (long)b * d.sCb;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int m = m0 + wm * 32 + p * 8 + g;
        if (m >= d.M) continue;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int n = n0 + wn * 16 + q * 8 + 2 * tg + h;
                if (n >= d.N) continue;
                double v = acc[p][q][h];
                if (d.scale_mode == 1) v = v * d.scale;
                else if (d.scale_mode == 2) v = v / d.scale;
                Cb[(long)m * d.sCm + (long)n * d.sCn] = v;
            }
        }
    }
}
static __global__ void __launch_bounds__(256) k_gemm_dmma(GemmDesc d, const double* __restrict__ A,
                                                   const double* __restrict__ B, double* __restrict__ C)
{
    k_gemm_dmma_run(blockIdx, gridDim, d, A, B, C);
}
struct k_gemm_dmma_b {
    static constexpr auto run = &k_gemm_dmma_run;
    static constexpr int maxt = 256, minb = 0;
};


// Split-TF32 contraction for the precision form: each FP32 operand is split
// into a TF32 head and a TF32 tail (x = hi + lo, hi = rna_tf32(x),
// lo = rna_tf32(x - hi)) and the product is hi*hi + hi*lo + lo*hi on the
// tensor cores (mma.sync m16n8k8 .tf32, FP32 accumulation), the 3-term
// compensated form that carries FP32-level accuracy through TF32 inputs.
// 64x64 block tile, 8 warps as 2 (m) x 4 (n), each warp 32x16 (2 x 2
// m16n8 fragments); k tiles of 16 through shared memory.
__device__ __forceinline__ uint32_t f32_to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo)
{
    hi = f32_to_tf32(x);
    lo = f32_to_tf32(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32_16x8x8(float* d, const uint32_t* a, const uint32_t* b)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

static __device__ __forceinline__ void k_gemm_tf32x3_run(const uint3 blockIdx, const dim3 gridDim,
    GemmDesc d, const float* __restrict__ A,
                                                            const float* __restrict__ B, float* __restrict__ C)
{
    constexpr int TM = 64, TN = 64, TK = 16, PAD = 8;
    __shared__ float As[TK][TM + PAD];
    __shared__ float Bs[TK][TN + PAD];
    const int b = blockIdx.z;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp >> 2, wn = warp & 3;
    const int g = lane >> 2, tg = lane & 3;
    const float* Ab = A + (long)b * d.sAb;
    const float* Bb = B + (long)b * d.sBb;
    float acc[2][2][4];
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[p][q][e] = 0.f;
    for (int k0 = 0; k0 < d.K; k0 += TK) {
        for (int t = threadIdx.x; t < TK * TM; t += 256) {
            const int kk = d.sAk == 1 ? t % TK : t / TM, mm = d.sAk == 1 ? t / TK : t % TM;
            const int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < d.M && k < d.K) ? Ab[(long)m * d.sAm + (long)k * d.sAk] : 0.f;
        }
        for (int t = threadIdx.x; t < TK * TN; t += 256) {
            const int kk = d.sBk == 1 ? t % TK : t / TN, nn = d.sBk == 1 ? t / TK : t % TN;
            const int n = n0 + nn, k = k0 + kk;
            Bs[kk][nn] = (n < d.N && k < d.K) ? Bb[(long)k * d.sBk + (long)n * d.sBn] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; kk += 8) {
            uint32_t ah[2][4], al[2][4], bh[2][2], bl[2][2];
#pragma unroll
            for (int p = 0; p < 2; ++p) {
                const int mr = wm * 32 + p * 16 + g;
                split_tf32(As[kk + tg][mr], ah[p][0], al[p][0]);
                split_tf32(As[kk + tg][mr + 8], ah[p][1], al[p][1]);
                split_tf32(As[kk + tg + 4][mr], ah[p][2], al[p][2]);
                split_tf32(As[kk + tg + 4][mr + 8], ah[p][3], al[p][3]);
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int nc = wn * 16 + q * 8 + g;
                split_tf32(Bs[kk + tg][nc], bh[q][0], bl[q][0]);
                split_tf32(Bs[kk + tg + 4][nc], bh[q][1], bl[q][1]);
            }
#pragma unroll
            for (int p = 0; p < 2; ++p)
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    mma_tf32_16x8x8(acc[p][q], al[p], bh[q]);
                    mma_tf32_16x8x8(acc[p][q], ah[p], bl[q]);
                    mma_tf32_16x8x8(acc[p][q], ah[p], bh[q]);
                }
        }
        __syncthreads();
    }
    float* Cb = C + (long)b * d.sCb;
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int m = m0 + wm * 32 + p * 16 + g + (e >= 2 ? 8 : 0);
                const int n = n0 + wn * 16 + q * 8 + 2 * tg + (e & 1);
                if (m >= d.M || n >= d.N) continue;
                float v = acc[p][q][e];
                if (d.scale_mode == 1) v = v * (float)d.scale;
                else if (d.scale_mode == 2) v = v / (float)d.scale;
                Cb[(long)m * d.sCm + (long)n * d.sCn] = v;
            }
}
static __global__ void __launch_bounds__(256) k_gemm_tf32x3(GemmDesc d, const float* __restrict__ A,
                                                            const float* __restrict__ B, float* __restrict__ C)
{
    k_gemm_tf32x3_run(blockIdx, gridDim, d, A, B, C);
}
struct k_gemm_tf32x3_b {
    static constexpr auto run = &k_gemm_tf32x3_run;
    static constexpr int maxt = 256, minb = 0;
};

}  // namespace
}  // namespace pll
