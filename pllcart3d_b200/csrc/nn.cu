// Kernels of the learned surrogate (a 3-d convolutional U-Net that advances
// the cell-centred state of a fingering run by 8 steps): forward, backward
// and Adam, hand-written for the BF16 tensor cores (mma.sync m16n8k16, BF16
// operands, FP32 accumulation).
//
// The forward convolution (and so the input gradient) runs on the 5th-
// generation tensor cores where the shapes allow (nn_umma.cuh: tcgen05.mma
// with a TMEM accumulator, TMA-staged operands whose out-of-bounds fill is
// the zero padding), else on the mma.sync kernel below.
//
// Layout: activations are channels-last [n][d][h][w][c] (voxel-major, c
// contiguous), BF16 as operands of the convolutions, FP32 for
// pre-activations and gradients that are accumulated.  Weights are
// [cout][tap][cin] with tap = (dz*3 + dy)*3 + dx.
//
//  * 3x3x3 (and 1x1x1) convolution, zero padding, stride 1, as an implicit
//    GEMM: rows = voxels (128 per CTA), columns = output channels, K = taps x
//    input channels in chunks of 16; the shifted input rows are gathered
//    straight from global memory (16-byte loads, zero outside the volume),
//    double-buffered through shared memory, bias and leaky-ReLU fused in the
//    epilogue.
//  * the input gradient is the same convolution of the output gradient with
//    the weights flipped in space and transposed in channels;
//  * the weight gradient is a GEMM over voxels (cout x cin per tap), split
//    over voxel chunks, FP32 atomics into the gradient;
//  * 2x average pooling, 2x nearest upsampling, channel concatenation,
//    activation backward with the bias-gradient reduction, MSE loss, Adam.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "nn_umma.cuh"

typedef __nv_bfloat16 bf16;

namespace {

struct Vol {
    int N, D, H, W;
};

__device__ __forceinline__ void mma16816(float* c, const uint32_t* a, const uint32_t* b)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float leaky(float x, float slope) { return x > 0.f ? x : slope * x; }

constexpr int CBM = 128;   // voxels per CTA
constexpr int CBK = 16;    // K chunk (input channels of one tap)
constexpr int CPAD = 24;   // shared row pitch in bf16 (48 bytes: conflict-free fragments)

// Y = act(conv(X, W) + bias): Y32 (pre-activation, FP32) and/or Y16 (post,
// BF16); Cin % 16 == 0, pointers 16-byte aligned
template <int BN>
__global__ void __launch_bounds__(256) k_conv_fwd(const bf16* __restrict__ X, Vol g, int Cin,
                                                  const bf16* __restrict__ Wt, const float* __restrict__ bias,
                                                  int Cout, int ksize, float* __restrict__ Y32,
                                                  bf16* __restrict__ Y16, int act, float slope)
{
    __shared__ __align__(16) bf16 As[2][CBM][CPAD];
    __shared__ __align__(16) bf16 Bs[2][BN][CPAD];
    const long V = (long)g.N * g.D * g.H * g.W;
    const long m0 = (long)blockIdx.x * CBM;
    const int n0 = blockIdx.y * BN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int gq = lane >> 2, tq = lane & 3;
    constexpr int WN = BN / 2;      // warp tile columns
    constexpr int NQ = WN / 8;      // n8 fragments per warp

    // A loader: row ar (voxel), 8 channels (half ah of the 16-chunk)
    const int ar = tid >> 1, ah = tid & 1;
    const long av = m0 + ar;
    const bool avalid = av < V;
    int an = 0, ad = 0, ahh = 0, aw = 0;
    if (avalid) {
        long t = av;
        aw = (int)(t % g.W);
        t /= g.W;
        ahh = (int)(t % g.H);
        t /= g.H;
        ad = (int)(t % g.D);
        an = (int)(t / g.D);
    }
    const int br = tid >> 1, bh = tid & 1;
    const int ntaps = ksize * ksize * ksize;
    const int kchunks = Cin / CBK;
    const int nk = ntaps * kchunks;

    float acc[2][NQ][4];
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[p][q][e] = 0.f;

    uint4 ra, rb;
    auto load = [&](int kk) {
        const int tap = kk / kchunks, c0 = (kk - tap * kchunks) * CBK;
        int dz = 0, dy = 0, dx = 0;
        if (ksize == 3) {
            dz = tap / 9 - 1;
            dy = (tap / 3) % 3 - 1;
            dx = tap % 3 - 1;
        }
        ra = make_uint4(0, 0, 0, 0);
        const int d2 = ad + dz, h2 = ahh + dy, w2 = aw + dx;
        if (avalid && d2 >= 0 && d2 < g.D && h2 >= 0 && h2 < g.H && w2 >= 0 && w2 < g.W) {
            const long nv = (((long)an * g.D + d2) * g.H + h2) * g.W + w2;
            ra = *(const uint4*)(X + nv * Cin + c0 + 8 * ah);
        }
        rb = make_uint4(0, 0, 0, 0);
        if (tid < BN * 2) {
            const int co = n0 + br;
            if (co < Cout) rb = *(const uint4*)(Wt + ((long)co * ntaps + tap) * Cin + c0 + 8 * bh);
        }
    };
    load(0);
    for (int kk = 0; kk < nk; ++kk) {
        const int s = kk & 1;
        *(uint4*)&As[s][ar][8 * ah] = ra;
        if (tid < BN * 2) *(uint4*)&Bs[s][br][8 * bh] = rb;
        __syncthreads();
        if (kk + 1 < nk) load(kk + 1);
        uint32_t a[2][4], b[NQ][2];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const int r = wm * 32 + p * 16 + gq;
            a[p][0] = *(const uint32_t*)&As[s][r][2 * tq];
            a[p][1] = *(const uint32_t*)&As[s][r + 8][2 * tq];
            a[p][2] = *(const uint32_t*)&As[s][r][2 * tq + 8];
            a[p][3] = *(const uint32_t*)&As[s][r + 8][2 * tq + 8];
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int cn = wn * WN + q * 8 + gq;
            b[q][0] = *(const uint32_t*)&Bs[s][cn][2 * tq];
            b[q][1] = *(const uint32_t*)&Bs[s][cn][2 * tq + 8];
        }
#pragma unroll
        for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int q = 0; q < NQ; ++q) mma16816(acc[p][q], a[p], b[q]);
    }
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long row = m0 + wm * 32 + p * 16 + gq + 8 * h;
                const int col = n0 + wn * WN + q * 8 + 2 * tq;
                if (row >= V) continue;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    if (col + e >= Cout) continue;
                    float v = acc[p][q][2 * h + e] + (bias ? bias[col + e] : 0.f);
                    if (Y32) Y32[row * Cout + col + e] = v;
                    if (act) v = leaky(v, slope);
                    if (Y16) Y16[row * Cout + col + e] = __float2bfloat16(v);
                }
            }
}

// dW[co][tap][ci] += sum over voxels of G[v][co] * X[v + o(tap)][ci]
__global__ void __launch_bounds__(256) k_conv_wgrad(const bf16* __restrict__ G, const bf16* __restrict__ X,
                                                    Vol g, int Cin, int Cout, int ksize, long vchunk,
                                                    float* __restrict__ dW)
{
    __shared__ __align__(16) bf16 As[64][CPAD];   // [co][voxel]
    __shared__ __align__(16) bf16 Bs[64][CPAD];   // [ci][voxel]
    const long V = (long)g.N * g.D * g.H * g.W;
    const long v0 = (long)blockIdx.x * vchunk;
    const long v1 = v0 + vchunk < V ? v0 + vchunk : V;
    const int tap = blockIdx.y;
    const int ntc = (Cin + 63) / 64;
    const int co0 = (blockIdx.z / ntc) * 64, ci0 = (blockIdx.z % ntc) * 64;
    const int ntaps = ksize * ksize * ksize;
    int dz = 0, dy = 0, dx = 0;
    if (ksize == 3) {
        dz = tap / 9 - 1;
        dy = (tap / 3) % 3 - 1;
        dx = tap % 3 - 1;
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;   // warp tile 16 (co) x 32 (ci)
    const int gq = lane >> 2, tq = lane & 3;
    float acc[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[q][e] = 0.f;
    // loaders: threads 0-127 read 16 voxels x 64 output channels of G,
    // threads 128-255 the same voxels' shifted inputs, 8 channels each
    const int lr = (tid & 127) >> 3, lc = (tid & 7) * 8;
    for (long vb = v0; vb < v1; vb += 16) {
        const long v = vb + lr;
        bf16 vals[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) vals[e] = __float2bfloat16(0.f);
        if (v < v1) {
            if (tid < 128) {
                if (co0 + lc < Cout) {
                    const uint4 u = *(const uint4*)(G + v * Cout + co0 + lc);
                    const bf16* pv = (const bf16*)&u;
#pragma unroll
                    for (int e = 0; e < 8; ++e) vals[e] = pv[e];
                }
            } else {
                long t = v;
                const int w = (int)(t % g.W);
                t /= g.W;
                const int h = (int)(t % g.H);
                t /= g.H;
                const int d = (int)(t % g.D);
                const int n = (int)(t / g.D);
                const int d2 = d + dz, h2 = h + dy, w2 = w + dx;
                if (ci0 + lc < Cin && d2 >= 0 && d2 < g.D && h2 >= 0 && h2 < g.H && w2 >= 0 && w2 < g.W) {
                    const long nv = (((long)n * g.D + d2) * g.H + h2) * g.W + w2;
                    const uint4 u = *(const uint4*)(X + nv * Cin + ci0 + lc);
                    const bf16* pv = (const bf16*)&u;
#pragma unroll
                    for (int e = 0; e < 8; ++e) vals[e] = pv[e];
                }
            }
        }
        __syncthreads();   // previous chunk's fragments are consumed
        if (tid < 128) {
#pragma unroll
            for (int e = 0; e < 8; ++e) As[lc + e][lr] = vals[e];
        } else {
#pragma unroll
            for (int e = 0; e < 8; ++e) Bs[lc + e][lr] = vals[e];
        }
        __syncthreads();
        uint32_t a[4], b[4][2];
        const int r = wm * 16 + gq;
        a[0] = *(const uint32_t*)&As[r][2 * tq];
        a[1] = *(const uint32_t*)&As[r + 8][2 * tq];
        a[2] = *(const uint32_t*)&As[r][2 * tq + 8];
        a[3] = *(const uint32_t*)&As[r + 8][2 * tq + 8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int cn = wn * 32 + q * 8 + gq;
            b[q][0] = *(const uint32_t*)&Bs[cn][2 * tq];
            b[q][1] = *(const uint32_t*)&Bs[cn][2 * tq + 8];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) mma16816(acc[q], a, b[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int co = co0 + wm * 16 + gq + (e >= 2 ? 8 : 0);
            const int ci = ci0 + wn * 32 + q * 8 + 2 * tq + (e & 1);
            if (co < Cout && ci < Cin) atomicAdd(&dW[((long)co * ntaps + tap) * Cin + ci], acc[q][e]);
        }
}

// Wf[ci][t][co] = W[co][ntaps-1-t][ci]
__global__ void k_flip(const bf16* __restrict__ W, int Cout, int ntaps, int Cin, bf16* __restrict__ Wf)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long n = (long)Cout * ntaps * Cin;
    if (i >= n) return;
    const int ci = (int)(i % Cin);
    const int t = (int)((i / Cin) % ntaps);
    const int co = (int)(i / ((long)Cin * ntaps));
    Wf[((long)ci * ntaps + (ntaps - 1 - t)) * Cout + co] = W[i];
}

// dZ = dY * act'(Z) as BF16, and db[c] += sum_v dZ[v][c]
__global__ void k_act_bwd(const float* __restrict__ dY, const float* __restrict__ Z, long V, int C, int act,
                          float slope, bf16* __restrict__ dZ, float* __restrict__ db)
{
    // block: 256 threads over (voxel chunk, channels); one channel per
    // thread column, voxels strided
    const int c = blockIdx.y * 32 + (threadIdx.x & 31);
    const int vr = threadIdx.x >> 5;   // 0..7
    float s = 0.f;
    if (c < C) {
        for (long v = (long)blockIdx.x * 8 + vr; v < V; v += (long)gridDim.x * 8) {
            float gv = dY[v * C + c];
            if (act && Z[v * C + c] <= 0.f) gv *= slope;
            dZ[v * C + c] = __float2bfloat16(gv);
            s += gv;
        }
    }
    __shared__ float red[8][33];
    red[vr][threadIdx.x & 31] = s;
    __syncthreads();
    if (vr == 0 && c < C) {
        float t = 0.f;
        for (int r = 0; r < 8; ++r) t += red[r][threadIdx.x & 31];
        if (db) atomicAdd(&db[c], t);
    }
}

// 2x average pooling of X[N][D][H][W][C] (BF16 in and out)
__global__ void k_pool_fwd(const bf16* __restrict__ X, Vol g, int C, bf16* __restrict__ Y)
{
    const int D2 = g.D / 2, H2 = g.H / 2, W2 = g.W / 2;
    const long n = (long)g.N * D2 * H2 * W2 * C;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = (int)(i % C);
    long t = i / C;
    const int w = (int)(t % W2);
    t /= W2;
    const int h = (int)(t % H2);
    t /= H2;
    const int d = (int)(t % D2);
    const int b = (int)(t / D2);
    float s = 0.f;
    for (int a = 0; a < 8; ++a) {
        const long v = (((long)b * g.D + 2 * d + (a >> 2)) * g.H + 2 * h + ((a >> 1) & 1)) * g.W + 2 * w + (a & 1);
        s += __bfloat162float(X[v * C + c]);
    }
    Y[i] = __float2bfloat16(0.125f * s);
}

// gradient of the pooling into dX (FP32, X's volume g), accumulating when acc
__global__ void k_pool_bwd(const float* __restrict__ dY, Vol g, int C, float* __restrict__ dX, int acc)
{
    const long n = (long)g.N * g.D * g.H * g.W * C;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = (int)(i % C);
    long t = i / C;
    const int w = (int)(t % g.W);
    t /= g.W;
    const int h = (int)(t % g.H);
    t /= g.H;
    const int d = (int)(t % g.D);
    const int b = (int)(t / g.D);
    const long j = ((((long)b * (g.D / 2) + d / 2) * (g.H / 2) + h / 2) * (g.W / 2) + w / 2) * C + c;
    const float v = 0.125f * dY[j];
    dX[i] = acc ? dX[i] + v : v;
}

// 2x nearest upsampling of X (volume g) into Y (volume 2g)
__global__ void k_up_fwd(const bf16* __restrict__ X, Vol g, int C, bf16* __restrict__ Y)
{
    const long n = (long)g.N * (2 * g.D) * (2 * g.H) * (2 * g.W) * C;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = (int)(i % C);
    long t = i / C;
    const int w = (int)(t % (2 * g.W));
    t /= (2 * g.W);
    const int h = (int)(t % (2 * g.H));
    t /= (2 * g.H);
    const int d = (int)(t % (2 * g.D));
    const int b = (int)(t / (2 * g.D));
    Y[i] = X[((((long)b * g.D + d / 2) * g.H + h / 2) * g.W + w / 2) * C + c];
}

// gradient of the upsampling: dX (volume g) = sum of the 8 children
__global__ void k_up_bwd(const float* __restrict__ dY, Vol g, int C, float* __restrict__ dX, int acc)
{
    const long n = (long)g.N * g.D * g.H * g.W * C;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = (int)(i % C);
    long t = i / C;
    const int w = (int)(t % g.W);
    t /= g.W;
    const int h = (int)(t % g.H);
    t /= g.H;
    const int d = (int)(t % g.D);
    const int b = (int)(t / g.D);
    float s = 0.f;
    for (int a = 0; a < 8; ++a) {
        const long v = (((long)b * 2 * g.D + 2 * d + (a >> 2)) * 2 * g.H + 2 * h + ((a >> 1) & 1)) * 2 * g.W + 2 * w +
                       (a & 1);
        s += dY[v * C + c];
    }
    dX[i] = acc ? dX[i] + s : s;
}

// Y[v] = [A[v] (CA channels) | B[v] (CB channels)]
__global__ void k_cat_fwd(const bf16* __restrict__ A, int CA, const bf16* __restrict__ B, int CB, long V,
                          bf16* __restrict__ Y)
{
    const int C = CA + CB;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V * C) return;
    const long v = i / C;
    const int c = (int)(i % C);
    Y[i] = c < CA ? A[v * CA + c] : B[v * CB + (c - CA)];
}

__global__ void k_cat_bwd(const float* __restrict__ dY, int CA, int CB, long V, float* __restrict__ dA, int accA,
                          float* __restrict__ dB, int accB)
{
    const int C = CA + CB;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V * C) return;
    const long v = i / C;
    const int c = (int)(i % C);
    const float g = dY[i];
    if (c < CA) {
        if (dA) dA[v * CA + c] = accA ? dA[v * CA + c] + g : g;
    } else {
        if (dB) dB[v * CB + c - CA] = accB ? dB[v * CB + c - CA] + g : g;
    }
}

// loss += scale * sum (p - t)^2 ; grad = 2 scale (p - t)
__global__ void k_mse(const float* __restrict__ P, const float* __restrict__ T, long n, float scale,
                      float* __restrict__ grad, float* __restrict__ loss)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    float s = 0.f;
    if (i < n) {
        const float d = P[i] - T[i];
        if (grad) grad[i] = 2.f * scale * d;
        s = scale * d * d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, s);
}

// sum of squares of x into *out (global gradient norm for clipping)
__global__ void k_sumsq(const float* __restrict__ x, long n, float* __restrict__ out)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    float s = i < n ? x[i] * x[i] : 0.f;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// Adam (Kingma & Ba 2015) on FP32 master weights, BF16 copy out; with
// sumsq given, the gradient is scaled by min(1, clip / ||g||) (global norm
// clipping) and a non-finite norm skips the update
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, long n, float lr, float b1, float b2, float eps, float bc1, float bc2,
                       bf16* __restrict__ w16, const float* __restrict__ sumsq, float clip)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float scale = 1.f;
    if (sumsq) {
        const float nrm = sqrtf(*sumsq);
        if (!isfinite(nrm)) return;
        if (nrm > clip) scale = clip / nrm;
    }
    const float gi = g[i] * scale;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16(wi);
}

__global__ void k_cast(const float* __restrict__ x, long n, bf16* __restrict__ y)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

// network input: cell-centred (u, v, w, c) FP32 [V][4] of one sample plus
// the constant channels -> BF16 [V][16]: (c, u, v, w, r, p, 0 ... 0) after
// the per-channel affine normalisation (x - mean) / std
__global__ void k_pack_input(const float* __restrict__ cells, long V, float r, float p,
                             const float* __restrict__ norm /* mean[4], std[4] */, bf16* __restrict__ out)
{
    const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const float4 q = ((const float4*)cells)[v];   // u, v, w, c
    const float ch[4] = {q.w, q.x, q.y, q.z};       // c, u, v, w
    bf16* o = out + v * 16;
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = __float2bfloat16((ch[k] - norm[k]) / norm[4 + k]);
    o[4] = __float2bfloat16(r);
    o[5] = __float2bfloat16(p);
#pragma unroll
    for (int k = 6; k < 16; ++k) o[k] = __float2bfloat16(0.f);
}

// training target: the 8-step change of (c, u, v, w) over its scale,
// [V][16] with channels 4-15 zero
__global__ void k_pack_target(const float* __restrict__ a, const float* __restrict__ b, long V,
                              const float* __restrict__ scale /* c, u, v, w */, float* __restrict__ out)
{
    const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const float4 p = ((const float4*)a)[v], q = ((const float4*)b)[v];   // u, v, w, c
    float* o = out + v * 16;
    o[0] = (q.w - p.w) / scale[0];
    o[1] = (q.x - p.x) / scale[1];
    o[2] = (q.y - p.y) / scale[2];
    o[3] = (q.z - p.z) / scale[3];
#pragma unroll
    for (int k = 4; k < 16; ++k) o[k] = 0.f;
}

// prediction: cells + scale * out[:, 0:4] (out channels c, u, v, w)
__global__ void k_apply_delta(const float* __restrict__ a, const float* __restrict__ out, long V,
                              const float* __restrict__ scale, float* __restrict__ b)
{
    const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const float4 p = ((const float4*)a)[v];
    const float* o = out + v * 16;
    float4 q;
    q.w = p.w + scale[0] * o[0];
    q.x = p.x + scale[1] * o[1];
    q.y = p.y + scale[2] * o[2];
    q.z = p.z + scale[3] * o[3];
    ((float4*)b)[v] = q;
}

inline unsigned nblk(long n, int b) { return (unsigned)((n + b - 1) / b); }

// ---- the tcgen05 convolution: tensor maps, shape checks, dispatch ----------
int g_conv_path = 0;   // 0: tcgen05 where the shapes allow, 1: mma.sync, 2: tcgen05 or fail

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn nn_encode()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// the geometry of the tcgen05 path, false when the shapes do not fit it:
// tiles of 128 voxels made of whole w rows (W divides 128), hb rows of h and
// db slices of d; Cout a multiple of the column tile; Cin a multiple of 16
bool cu_geom(int N, int D, int H, int W, int Cin, int Cout, int ksize, CuGeom& g, int& BN, int& CK)
{
    const long V = (long)N * D * H * W;
    if (V % CU_BM || W > CU_BM || CU_BM % W || Cin % 16 || Cout % 16) return false;
    const int hb = (CU_BM / W) < H ? (CU_BM / W) : H;
    if (H % hb || (CU_BM / W) % hb) return false;
    const int db = CU_BM / (W * hb);
    if (db > D || D % db) return false;
    BN = Cout >= 128 ? 128 : Cout >= 64 ? 64 : Cout >= 32 ? 32 : 16;
    if (Cout % BN) return false;
    CK = Cin % 64 == 0 ? 64 : Cin % 32 == 0 ? 32 : 16;
    g = CuGeom{N, D, H, W, hb, db, Cin, Cout, ksize};
    return true;
}

bool cu_maps(const CuGeom& g, int BN, int CK, const void* X, const void* Wt, CUtensorMap* mx, CUtensorMap* mw)
{
    EncodeTiledFn fn = nn_encode();
    if (!fn) return false;
    const CUtensorMapSwizzle sw = CK == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                : CK == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
    const cuuint64_t c2 = (cuuint64_t)g.Cin * 2;
    const cuuint64_t xd[5] = {(cuuint64_t)g.Cin, (cuuint64_t)g.W, (cuuint64_t)g.H, (cuuint64_t)g.D, (cuuint64_t)g.N};
    const cuuint64_t xs[4] = {c2, c2 * g.W, c2 * g.W * g.H, c2 * g.W * g.H * g.D};
    const cuuint32_t xb[5] = {(cuuint32_t)CK, (cuuint32_t)g.W, (cuuint32_t)g.hb, (cuuint32_t)g.db, 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    if (fn(mx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void*)X, xd, xs, xb, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    const int taps = g.ksize * g.ksize * g.ksize;
    const cuuint64_t wd[3] = {(cuuint64_t)g.Cin, (cuuint64_t)taps, (cuuint64_t)g.Cout};
    const cuuint64_t ws[2] = {c2, c2 * taps};
    const cuuint32_t wb[3] = {(cuuint32_t)CK, 1, (cuuint32_t)BN};
    return fn(mw, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, (void*)Wt, wd, ws, wb, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, int CK>
bool cu_launch(const CUtensorMap& mx, const CUtensorMap& mw, const CuGeom& g, const float* bias, float* Y32,
               void* Y16, int act, float slope, cudaStream_t st)
{
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_conv_umma<BN, CK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)CuSmem<BN, CK>::DYN) != cudaSuccess)
            return false;
        attr = true;
    }
    const long V = (long)g.N * g.D * g.H * g.W;
    const dim3 grid((unsigned)(V / CU_BM), (unsigned)(g.Cout / BN));
    k_conv_umma<BN, CK><<<grid, CU_THREADS, CuSmem<BN, CK>::DYN, st>>>(mx, mw, g, bias, Y32, (__nv_bfloat16*)Y16,
                                                                         act, slope);
    return true;
}

template <int BN>
bool cu_launch_ck(int CK, const CUtensorMap& mx, const CUtensorMap& mw, const CuGeom& g, const float* bias,
                  float* Y32, void* Y16, int act, float slope, cudaStream_t st)
{
    if (CK == 64) return cu_launch<BN, 64>(mx, mw, g, bias, Y32, Y16, act, slope, st);
    if (CK == 32) return cu_launch<BN, 32>(mx, mw, g, bias, Y32, Y16, act, slope, st);
    return cu_launch<BN, 16>(mx, mw, g, bias, Y32, Y16, act, slope, st);
}

// the forward convolution on tcgen05; false when the shapes or the tensor
// maps do not fit (the caller then runs the mma.sync kernel)
bool conv_umma(const void* X, int N, int D, int H, int W, int Cin, const void* Wt, const float* bias, int Cout,
               int ksize, float* Y32, void* Y16, int act, float slope, cudaStream_t st)
{
    CuGeom g;
    int BN = 0, CK = 0;
    if (!cu_geom(N, D, H, W, Cin, Cout, ksize, g, BN, CK)) return false;
    if (((uintptr_t)Y32 & 15) || ((uintptr_t)Y16 & 15) || ((uintptr_t)bias & 3)) return false;
    CUtensorMap mx, mw;
    std::memset(&mx, 0, sizeof(mx));
    std::memset(&mw, 0, sizeof(mw));
    if (!cu_maps(g, BN, CK, X, Wt, &mx, &mw)) return false;
    if (BN == 128) return cu_launch_ck<128>(CK, mx, mw, g, bias, Y32, Y16, act, slope, st);
    if (BN == 64) return cu_launch_ck<64>(CK, mx, mw, g, bias, Y32, Y16, act, slope, st);
    if (BN == 32) return cu_launch_ck<32>(CK, mx, mw, g, bias, Y32, Y16, act, slope, st);
    return cu_launch_ck<16>(CK, mx, mw, g, bias, Y32, Y16, act, slope, st);
}

}  // namespace

extern "C" {

// status: 0 ok, 6 invalid argument (shapes), 2 launch failure
int pllnn_conv_fwd(const void* X, int N, int D, int H, int W, int Cin, const void* Wt, const float* bias, int Cout,
                   int ksize, float* Y32, void* Y16, int act, float slope, void* stream)
{
    if (Cin % 16 || (ksize != 1 && ksize != 3) || ((uintptr_t)X & 15) || ((uintptr_t)Wt & 15)) return 6;
    const Vol g{N, D, H, W};
    const long V = (long)N * D * H * W;
    cudaStream_t st = (cudaStream_t)stream;
    if (g_conv_path != 1 && conv_umma(X, N, D, H, W, Cin, Wt, bias, Cout, ksize, Y32, Y16, act, slope, st))
        return cudaGetLastError() == cudaSuccess ? 0 : 2;
    if (g_conv_path == 2) return 6;
    if (Cout <= 32) {
        dim3 grid(nblk(V, CBM), nblk(Cout, 32));
        k_conv_fwd<32><<<grid, 256, 0, st>>>((const bf16*)X, g, Cin, (const bf16*)Wt, bias, Cout, ksize, Y32,
                                             (bf16*)Y16, act, slope);
    } else {
        dim3 grid(nblk(V, CBM), nblk(Cout, 64));
        k_conv_fwd<64><<<grid, 256, 0, st>>>((const bf16*)X, g, Cin, (const bf16*)Wt, bias, Cout, ksize, Y32,
                                             (bf16*)Y16, act, slope);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// which kernel the forward convolution uses: 0 the tcgen05 kernel where the
// shapes allow (default), 1 the mma.sync kernel, 2 the tcgen05 kernel or
// status 6; returns the previous setting
int pllnn_set_conv_path(int path)
{
    const int old = g_conv_path;
    if (path >= 0 && path <= 2) g_conv_path = path;
    return old;
}

// the library's status bits (0x100: a bounded wait of the tcgen05
// convolution ran out), cleared by the read
int pllnn_status(void)
{
    int v = 0, z = 0;
    if (cudaMemcpyFromSymbol(&v, g_nn_status, sizeof(int)) != cudaSuccess) return -1;
    if (v) cudaMemcpyToSymbol(g_nn_status, &z, sizeof(int));
    return v;
}

int pllnn_conv_wgrad(const void* G, const void* X, int N, int D, int H, int W, int Cin, int Cout, int ksize,
                     float* dW, void* stream)
{
    if (Cin % 8 || Cout % 8 || (ksize != 1 && ksize != 3)) return 6;
    const Vol g{N, D, H, W};
    const long V = (long)N * D * H * W;
    const int ntaps = ksize * ksize * ksize;
    const int tiles = ((Cout + 63) / 64) * ((Cin + 63) / 64);
    long chunks = 4096 / ((long)ntaps * tiles);
    if (chunks < 1) chunks = 1;
    long vchunk = (V + chunks - 1) / chunks;
    vchunk = ((vchunk + 15) / 16) * 16;
    if (vchunk < 256) vchunk = 256;
    dim3 grid((unsigned)((V + vchunk - 1) / vchunk), ntaps, tiles);
    k_conv_wgrad<<<grid, 256, 0, (cudaStream_t)stream>>>((const bf16*)G, (const bf16*)X, g, Cin, Cout, ksize, vchunk,
                                                         dW);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_flip(const void* Wt, int Cout, int ntaps, int Cin, void* Wf, void* stream)
{
    const long n = (long)Cout * ntaps * Cin;
    k_flip<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)Wt, Cout, ntaps, Cin, (bf16*)Wf);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_act_bwd(const float* dY, const float* Z, long V, int C, int act, float slope, void* dZ, float* db,
                  void* stream)
{
    long bx = (V + 8 * 64 - 1) / (8 * 64);
    if (bx > 4096) bx = 4096;
    dim3 grid((unsigned)bx, (C + 31) / 32);
    k_act_bwd<<<grid, 256, 0, (cudaStream_t)stream>>>(dY, Z, V, C, act, slope, (bf16*)dZ, db);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_pool_fwd(const void* X, int N, int D, int H, int W, int C, void* Y, void* stream)
{
    if (D % 2 || H % 2 || W % 2) return 6;
    const long n = (long)N * (D / 2) * (H / 2) * (W / 2) * C;
    k_pool_fwd<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)X, Vol{N, D, H, W}, C, (bf16*)Y);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_pool_bwd(const float* dY, int N, int D, int H, int W, int C, float* dX, int acc, void* stream)
{
    const long n = (long)N * D * H * W * C;
    k_pool_bwd<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(dY, Vol{N, D, H, W}, C, dX, acc);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_up_fwd(const void* X, int N, int D, int H, int W, int C, void* Y, void* stream)
{
    const long n = (long)N * 8 * D * H * W * C;
    k_up_fwd<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)X, Vol{N, D, H, W}, C, (bf16*)Y);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_up_bwd(const float* dY, int N, int D, int H, int W, int C, float* dX, int acc, void* stream)
{
    const long n = (long)N * D * H * W * C;
    k_up_bwd<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(dY, Vol{N, D, H, W}, C, dX, acc);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_cat_fwd(const void* A, int CA, const void* B, int CB, long V, void* Y, void* stream)
{
    k_cat_fwd<<<nblk(V * (CA + CB), 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)A, CA, (const bf16*)B, CB, V,
                                                                         (bf16*)Y);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_cat_bwd(const float* dY, int CA, int CB, long V, float* dA, int accA, float* dB, int accB, void* stream)
{
    k_cat_bwd<<<nblk(V * (CA + CB), 256), 256, 0, (cudaStream_t)stream>>>(dY, CA, CB, V, dA, accA, dB, accB);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_mse(const float* P, const float* T, long n, float scale, float* grad, float* loss, void* stream)
{
    k_mse<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(P, T, n, scale, grad, loss);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_adam(float* w, const float* g, float* m, float* v, long n, float lr, float b1, float b2, float eps, int t,
               void* w16, const float* sumsq, float clip, void* stream)
{
    const float bc1 = 1.f - powf(b1, (float)t), bc2 = 1.f - powf(b2, (float)t);
    k_adam<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, b1, b2, eps, bc1, bc2, (bf16*)w16,
                                                           sumsq, clip);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_sumsq(const float* x, long n, float* out, void* stream)
{
    k_sumsq<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(x, n, out);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_cast(const float* x, long n, void* y, void* stream)
{
    k_cast<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(x, n, (bf16*)y);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_pack_input(const float* cells, long V, float r, float p, const float* norm, void* out, void* stream)
{
    k_pack_input<<<nblk(V, 256), 256, 0, (cudaStream_t)stream>>>(cells, V, r, p, norm, (bf16*)out);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_pack_target(const float* a, const float* b, long V, const float* scale, float* out, void* stream)
{
    k_pack_target<<<nblk(V, 256), 256, 0, (cudaStream_t)stream>>>(a, b, V, scale, out);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int pllnn_apply_delta(const float* a, const float* out, long V, const float* scale, float* b, void* stream)
{
    k_apply_delta<<<nblk(V, 256), 256, 0, (cudaStream_t)stream>>>(a, out, V, scale, b);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // extern "C"
