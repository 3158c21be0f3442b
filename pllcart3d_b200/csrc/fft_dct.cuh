// FFT form of the DCT passes of the Poisson solve (phisolver_dct,
// pllcart3d.c:2035, 2104 through fftw_3d.h:45-106): FFTW's REDFT10 (DCT-II)
// and REDFT01 (DCT-III), unnormalised as FFTW defines them, along one axis
// of a batch of lines, for power-of-two lengths 8 ... 256.
//
// Method (Makhoul, "A fast cosine transform in one and multiple dimensions",
// IEEE Trans. ASSP 28(1), 1980): the DCT-II of x is 2 Re(e^{-i pi k/(2N)}
// V_k) with V the length-N DFT of the reordering v_n = x_{2n},
// v_{N-1-n} = x_{2n+1}; the DCT-III runs the same steps backwards
// (V_k = e^{i pi k/(2N)} (x_k - i x_{N-k}), an inverse DFT, the inverse
// reordering).  Two real lines share one complex DFT (line a in the real
// part, line b in the imaginary part), split afterwards by the conjugate
// symmetry of real transforms.  The DFT is the four-step factorisation
// N = R1 x R2 (Cooley-Tukey): R2 DFTs of length R1 over stride-R2
// subsequences, twiddles W_N^{n2 k1}, R1 DFTs of length R2; each short DFT
// (R <= 16) runs in registers as a radix-2 recursion.
//
// HBM traffic: one read and one write of the array per pass (the dense
// contraction this replaces performs 2N flops per element and is bound by
// the FP64 tensor pipe; this one performs ~5 log2(N) flops per element and
// is bound by HBM).  Results agree with the dense contraction to rounding
// (the FFT's error grows as log N, the direct sum's as N).
#pragma once

#include <cuda_runtime.h>

namespace pll {
namespace {

template <typename real>
struct cplx {
    real re, im;
};

template <typename real>
__device__ __forceinline__ cplx<real> cadd(cplx<real> a, cplx<real> b) { return {a.re + b.re, a.im + b.im}; }
template <typename real>
__device__ __forceinline__ cplx<real> csub(cplx<real> a, cplx<real> b) { return {a.re - b.re, a.im - b.im}; }
template <typename real>
__device__ __forceinline__ cplx<real> cmul(cplx<real> a, real c, real s)   // a * (c + i s)
{
    return {a.re * c - a.im * s, a.re * s + a.im * c};
}

// cos / sin of 2 pi m / 16, m = 0 .. 4 (the twiddles of DFTs up to 16 points)
__device__ __forceinline__ double tw16c(int m)
{
    return m == 0 ? 1.0 : m == 1 ? 0.92387953251128675613 : m == 2 ? 0.70710678118654752440
                                                   : m == 3 ? 0.38268343236508977173 : 0.0;
}

// W_R^k = exp(SGN * 2 pi i k / R) for R <= 16, 0 <= k < R/2
template <int R, int SGN>
__device__ __forceinline__ void twiddle(int k, double& c, double& s)
{
    const int m = k * (16 / R);   // in sixteenths of a turn, 0 <= m < 8
    if (m <= 4) {
        c = tw16c(m);
        s = tw16c(4 - m);
    } else {
        c = -tw16c(8 - m);
        s = tw16c(m - 4);
    }
    s = SGN < 0 ? -s : s;
}

// in-place DFT of R points in natural order, X_k = sum_n v_n W_R^{nk},
// W_R = exp(SGN 2 pi i / R): radix-2 decimation in time, fully unrolled
template <typename real, int R, int SGN>
struct Dft {
    static __device__ __forceinline__ void run(cplx<real>* v)
    {
        cplx<real> e[R / 2], o[R / 2];
#pragma unroll
        for (int n = 0; n < R / 2; ++n) {
            e[n] = v[2 * n];
            o[n] = v[2 * n + 1];
        }
        Dft<real, R / 2, SGN>::run(e);
        Dft<real, R / 2, SGN>::run(o);
#pragma unroll
        for (int k = 0; k < R / 2; ++k) {
            double c, s;
            twiddle<R, SGN>(k, c, s);
            const cplx<real> t = k == 0 ? o[k] : cmul(o[k], (real)c, (real)s);
            v[k] = cadd(e[k], t);
            v[k + R / 2] = csub(e[k], t);
        }
    }
};

template <typename real, int SGN>
struct Dft<real, 1, SGN> {
    static __device__ __forceinline__ void run(cplx<real>*) {}
};

// the factorisation N = R1 x R2 used for each length
template <int N>
struct FftShape {
    static constexpr int R1 = N >= 256 ? 16 : N >= 128 ? 16 : N >= 64 ? 8 : N >= 32 ? 8 : 4;
    static constexpr int R2 = N / R1;
    static_assert(R1 * R2 == N && R2 >= 2 && R2 <= 16, "unsupported FFT length");
};

// Line set of one pass: line L = a * inner + b starts at a*sa + b*sb, its
// elements step by se.  CONTIG: se == 1 (lines along the contiguous axis);
// otherwise sb == 1 (neighbouring lines are neighbouring elements).
struct FftLines {
    int lines, inner;
    long sa_in, sb_in, se_in;
    long sa_out, sb_out, se_out;
    double scale;   // output multiplier
};

constexpr int FFT_PB = 8;            // complex line pairs per block
constexpr int FFT_THREADS = FFT_PB * 16;

template <int N>
struct FftRow {
    static constexpr int value = N + N / 16 + 1;   // padded complex row per pair
};

template <int N>
constexpr size_t fft_smem_bytes() { return sizeof(cplx<double>) * (size_t)FFT_PB * FftRow<N>::value; }

// padded shared-memory slot of position n in a pair's row
template <int N>
__device__ __forceinline__ int fslot(int n) { return n + (n >> 4); }

// Makhoul reordering: position j of the line <-> index n of v
template <int N>
__device__ __forceinline__ int mperm(int j) { return (j & 1) ? N - 1 - (j >> 1) : (j >> 1); }

// KIND 0: DCT-II (REDFT10); KIND 1: DCT-III (REDFT01).  2*FFT_PB
// consecutive lines per block (inner must be a multiple of 2*FFT_PB).
// tw: cos / sin of 2 pi m / N (m < N); wq: cos / sin of pi k / (2N) (k < N)
template <typename real, int N, int KIND, bool CONTIG>
__device__ __forceinline__ void k_dct_fft_run(const uint3 blockIdx, const dim3 gridDim,
    FftLines d, const real* __restrict__ in,
                                                         real* __restrict__ out, const double2* __restrict__ tw,
                                                         const double2* __restrict__ wq)
{
    constexpr int R1 = FftShape<N>::R1, R2 = FftShape<N>::R2, ROW = FftRow<N>::value;
    constexpr int TL = 2 * FFT_PB;   // real lines per block
    extern __shared__ __align__(16) unsigned char fsm[];
    cplx<real>* C = (cplx<real>*)fsm;
    const int tid = threadIdx.x;
    const long L0 = (long)blockIdx.x * TL;
    const long a = L0 / d.inner, b0 = L0 % d.inner;
    const real* gin = in + a * d.sa_in + b0 * d.sb_in;
    real* gout = out + a * d.sa_out + b0 * d.sb_out;

    // ---- load: line l of the tile -> pair l/2, real (even l) or imaginary
    // part; all of a thread's loads are issued before the first store to
    // shared memory (TL*N/FFT_THREADS = N/8 of them), so they overlap
    constexpr int LPT = TL * N / FFT_THREADS;
    {
        real v[LPT];
#pragma unroll
        for (int t = 0; t < LPT; ++t) {
            const int e = tid + t * FFT_THREADS;
            int l, p;
            if (CONTIG) { l = e / N; p = e % N; } else { p = e / TL; l = e % TL; }
            v[t] = CONTIG ? gin[(long)l * d.sb_in + p] : gin[l + (long)p * d.se_in];
        }
#pragma unroll
        for (int t = 0; t < LPT; ++t) {
            const int e = tid + t * FFT_THREADS;
            int l, p;
            if (CONTIG) { l = e / N; p = e % N; } else { p = e / TL; l = e % TL; }
            const int n = KIND == 0 ? mperm<N>(p) : p;
            real* slot = &C[(l >> 1) * ROW + fslot<N>(n)].re;
            slot[l & 1] = v[t];
        }
    }
    __syncthreads();

    if (KIND == 1) {
        // V_k = e^{i pi k/(2N)} [(a_k + b_{N-k}) + i (b_k - a_{N-k})] for k and N-k
        for (int t = tid; t < FFT_PB * (N / 2 + 1); t += FFT_THREADS) {
            const int q = t / (N / 2 + 1), k = t % (N / 2 + 1);
            cplx<real>* row = C + q * ROW;
            const int km = (N - k) & (N - 1);   // N-k, with x_N = 0 at k = 0
            const cplx<real> xk = row[fslot<N>(k)];
            const cplx<real> xm = k == 0 ? cplx<real>{(real)0, (real)0} : row[fslot<N>(km)];
            const double2 w = wq[k];
            row[fslot<N>(k)] = cmul(cplx<real>{xk.re + xm.im, xk.im - xm.re}, (real)w.x, (real)w.y);
            if (k != 0 && k != N / 2) {
                const double2 w2 = wq[km];
                row[fslot<N>(km)] = cmul(cplx<real>{xm.re + xk.im, xm.im - xk.re}, (real)w2.x, (real)w2.y);
            }
        }
        __syncthreads();
    }

    constexpr int SGN = KIND == 0 ? -1 : 1;
    // ---- pass 1: for each n2, DFT_R1 over v[n2 + R2 n1]; twiddle W_N^{n2 k1}
    for (int t = tid; t < FFT_PB * R2; t += FFT_THREADS) {
        const int q = t / R2, n2 = t % R2;
        cplx<real>* row = C + q * ROW;
        cplx<real> v[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) v[n1] = row[fslot<N>(n2 + R2 * n1)];
        Dft<real, R1, SGN>::run(v);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) {
            const int m = (n2 * k1) & (N - 1);
            const double2 w = tw[m];
            const cplx<real> r = m == 0 ? v[k1] : cmul(v[k1], (real)w.x, (real)(SGN * w.y));
            row[fslot<N>(n2 + R2 * k1)] = r;   // y[k1][n2]
        }
    }
    __syncthreads();
    // ---- pass 2: for each k1, DFT_R2 over y[k1][n2]; X[k1 + R1 k2]
    cplx<real> x[R2];
    const bool live2 = tid < FFT_PB * R1;
    const int q2 = tid / R1, k1 = tid % R1;
    if (live2) {
        const cplx<real>* row = C + q2 * ROW;
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) x[n2] = row[fslot<N>(n2 + R2 * k1)];
        Dft<real, R2, SGN>::run(x);
    }
    __syncthreads();
    if (live2) {
        cplx<real>* row = C + q2 * ROW;
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) row[fslot<N>(k1 + R1 * k2)] = x[k2];
    }
    __syncthreads();

    if (KIND == 0) {
        // Y^a_k = Re(w Z_k) + Re(w conj Z_{N-k}), Y^b_k = Im(w Z_k) - Im(w conj Z_{N-k}),
        // w = e^{-i pi k/(2N)}; k and N-k together, in place
        for (int t = tid; t < FFT_PB * (N / 2 + 1); t += FFT_THREADS) {
            const int q = t / (N / 2 + 1), k = t % (N / 2 + 1);
            cplx<real>* row = C + q * ROW;
            const int km = (N - k) & (N - 1);
            const cplx<real> zk = row[fslot<N>(k)], zm = row[fslot<N>(km)];
            const double2 w = wq[k];
            // w Z_k and w conj(Z_{N-k}) with w = (c, -s)
            const cplx<real> p1 = cmul(zk, (real)w.x, (real)-w.y);
            const cplx<real> p2 = cmul(cplx<real>{zm.re, -zm.im}, (real)w.x, (real)-w.y);
            const cplx<real> yk = {p1.re + p2.re, p1.im - p2.im};
            if (k != 0 && k != N / 2) {
                const double2 w2 = wq[km];
                const cplx<real> r1 = cmul(zm, (real)w2.x, (real)-w2.y);
                const cplx<real> r2 = cmul(cplx<real>{zk.re, -zk.im}, (real)w2.x, (real)-w2.y);
                row[fslot<N>(km)] = cplx<real>{r1.re + r2.re, r1.im - r2.im};
            }
            row[fslot<N>(k)] = yk;
        }
        __syncthreads();
    }

    // ---- store: DCT-II in natural order; DCT-III through the inverse reordering
    const real sc = (real)d.scale;
#pragma unroll 8
    for (int e = tid; e < TL * N; e += FFT_THREADS) {
        int l, p;
        if (CONTIG) { l = e / N; p = e % N; } else { p = e / TL; l = e % TL; }
        const int n = KIND == 0 ? p : mperm<N>(p);
        const real* slot = &C[(l >> 1) * ROW + fslot<N>(n)].re;
        const real v = slot[l & 1] * sc;
        if (CONTIG) gout[(long)l * d.sb_out + p] = v;
        else gout[l + (long)p * d.se_out] = v;
    }
}
template <typename real, int N, int KIND, bool CONTIG>
__global__ void __launch_bounds__(FFT_THREADS) k_dct_fft(FftLines d, const real* __restrict__ in,
                                                         real* __restrict__ out, const double2* __restrict__ tw,
                                                         const double2* __restrict__ wq)
{
    k_dct_fft_run<real, N, KIND, CONTIG>(blockIdx, gridDim, d, in, out, tw, wq);
}
template <typename real, int N, int KIND, bool CONTIG>
struct k_dct_fft_b {
    static constexpr auto run = &k_dct_fft_run<real, N, KIND, CONTIG>;
    static constexpr int maxt = FFT_THREADS, minb = 0;
};

}  // namespace
}  // namespace pll
