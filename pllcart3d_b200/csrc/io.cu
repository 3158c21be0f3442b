// Snapshot, restart and diagnostic outputs of the reference, produced from
// the device-resident state:
//
//   write_to_file  pllcart3d.c:3047-3092  caf%04dR%03d.bin, float32
//                  (u, v, w at cell centres, c) per interior cell, i-j-k
//                  order; above 2e7 cells only cells with even i, j, k
//   midfield       L3121-3178             middata (text) + midfield%03d.bin,
//                  14 FP64 fields row by row over the padded box
//   intermediate   L3181-3228             reads them back
//   conc_average   L3635-3728             cavgy.bin / cavgz.bin / cavgyz.bin
//   find_wmax      L3606-3632             wmax.bin
//   find_max       L3539-3603             Outscreen (max |u|,|v|,|w|,|c| and
//                                         where), NaN guard on c
//
// Device kernels gather each file's values into a compact buffer (cell-centre
// averages, row packing, the averages' sequential sums in the reference's
// order), one copy brings it to pinned host memory, the host writes it.  Byte
// formats, file names, append/overwrite modes and the printf formats are the
// reference's; the precision form widens its FP32 fields to FP64 first.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pllcart3d_gpu.h"
#include "forms.h"
#include "host_common.cuh"

using namespace pll;

namespace pll {
namespace {

// ---- device kernels ------------------------------------------------------------

// cell-centre (u, v, w, c) of the cells (i0 + st*a, j0 + st*b, k0 + st*c)
template <typename real>
__global__ void k_pack_caf(Geo G, const real* __restrict__ u, const real* __restrict__ v,
                           const real* __restrict__ w, const real* __restrict__ c, int i0, int j0, int k0,
                           int st, int ni, int nj, int nk, float* __restrict__ out)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long total = (long)ni * nj * nk;
    if (t >= total) return;
    const int a = (int)(t / ((long)nj * nk));
    const int rem = (int)(t % ((long)nj * nk));
    const int i = i0 + st * a, j = j0 + st * (rem / nk), k = k0 + st * (rem % nk);
    const long id = (long)i * G.sx + (long)j * G.sy + k;
    const double uval = 0.5 * ((double)u[id] + (double)u[id + G.sx]);
    const double vval = 0.5 * ((double)v[id] + (double)v[id + G.sy]);
    const double wval = 0.5 * ((double)w[id] + (double)w[id + 1]);
    out[4 * t + 0] = (float)uval;
    out[4 * t + 1] = (float)vval;
    out[4 * t + 2] = (float)wval;
    out[4 * t + 3] = (float)(double)c[id];
}

// the inverse for a learned model's prediction: cell-centred (u, v, w, c)
// back into c's interior (and its y/z Neumann ghosts, as the x sweep of
// concentration fills them) and the interior faces of u, v, w (the mean of
// the two adjacent cell centres); inlet, outlet and wall faces keep their
// values
template <typename real>
__global__ void k_unpack_cells(Geo G, Rng R, const float4* __restrict__ cells, real* __restrict__ c,
                               real* __restrict__ u, real* __restrict__ v, real* __restrict__ w)
{
    const int k = R.ks + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = R.js + blockIdx.y;
    const int i = R.is + blockIdx.z;
    if (k > R.ke) return;
    const int nj = R.je - R.js + 1, nk = R.ke - R.ks + 1;
    auto cell = [&](int ii, int jj, int kk) {
        return cells[((long)(ii - R.is) * nj + (jj - R.js)) * nk + (kk - R.ks)];
    };
    const long id = (long)i * G.sx + (long)j * G.sy + k;
    const float4 q = cell(i, j, k);
    const real cv = (real)q.w;
    c[id] = cv;
    if (j == R.js) c[id - G.sy] = cv;
    if (j == R.je) c[id + G.sy] = cv;
    if (k == R.ks) {
        c[id - 1] = cv;
        if (j == R.js) c[id - G.sy - 1] = cv;
        if (j == R.je) c[id + G.sy - 1] = cv;
    }
    if (k == R.ke) {
        c[id + 1] = cv;
        if (j == R.js) c[id - G.sy + 1] = cv;
        if (j == R.je) c[id + G.sy + 1] = cv;
    }
    if (i > R.is) u[id] = (real)(0.5f * (cell(i - 1, j, k).x + q.x));
    if (j > R.js) v[id] = (real)(0.5f * (cell(i, j - 1, k).y + q.y));
    if (k > R.ks) w[id] = (real)(0.5f * (cell(i, j, k - 1).z + q.z));
}

constexpr int NMID = 14;
template <typename real>
struct MidPtrs {
    real* f[NMID];
};

// midfield row packing for planes [ia, ib): out[((i-ia)*NY + j)*14 + f][k]
template <typename real>
__global__ void k_pack_mid(Geo G, MidPtrs<real> P, int ia, double* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = ia + blockIdx.z;
    if (k >= G.NZ) return;
    const long id = (long)i * G.sx + (long)j * G.sy + k;
    double* o = out + (((long)blockIdx.z * G.NY + j) * NMID) * G.NZ + k;
#pragma unroll
    for (int f = 0; f < NMID; ++f) o[(long)f * G.NZ] = (double)P.f[f][id];
}

template <typename real>
__global__ void k_unpack_mid(Geo G, MidPtrs<real> P, int ia, const double* __restrict__ in)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = ia + blockIdx.z;
    if (k >= G.NZ) return;
    const long id = (long)i * G.sx + (long)j * G.sy + k;
    const double* p = in + (((long)blockIdx.z * G.NY + j) * NMID) * G.NZ + k;
#pragma unroll
    for (int f = 0; f < NMID; ++f) P.f[f][id] = (real)p[(long)f * G.NZ];
}

// conc_average: y averages per (i,k), z averages per (i,j), sums in the
// reference's sequential order in FP64, divided by the cell count
template <typename real>
__global__ void k_cavg_y(Geo G, Rng R, const real* __restrict__ c, float* __restrict__ out)
{
    const int k = R.ks + blockIdx.x * blockDim.x + threadIdx.x;
    const int i = R.is + blockIdx.y;
    if (k > R.ke) return;
    double s = 0;
    for (int j = R.js; j <= R.je; ++j) s += (double)c[(long)i * G.sx + (long)j * G.sy + k];
    out[(long)(i - R.is) * (R.ke - R.ks + 1) + (k - R.ks)] = (float)(s / (R.je - R.js + 1));
}

template <typename real>
__global__ void k_cavg_z(Geo G, Rng R, const real* __restrict__ c, float* __restrict__ out)
{
    const int j = R.js + blockIdx.x * blockDim.x + threadIdx.x;
    const int i = R.is + blockIdx.y;
    if (j > R.je) return;
    const long b = (long)i * G.sx + (long)j * G.sy;
    double s = 0;
    for (int k = R.ks; k <= R.ke; ++k) s += (double)c[b + k];
    out[(long)(i - R.is) * (R.je - R.js + 1) + (j - R.js)] = (float)(s / (R.ke - R.ks + 1));
}

template <typename real>
__global__ void k_cavg_yz(Geo G, Rng R, const real* __restrict__ c, float* __restrict__ out)
{
    const int i = R.is + blockIdx.x * blockDim.x + threadIdx.x;
    if (i > R.ie) return;
    double s = 0;
    for (int j = R.js; j <= R.je; ++j) {
        const long b = (long)i * G.sx + (long)j * G.sy;
        for (int k = R.ks; k <= R.ke; ++k) s += (double)c[b + k];
    }
    out[i - R.is] = (float)(s / ((R.je - R.js + 1) * (R.ke - R.ks + 1)));
}

// max over the interior of w, starting from 0 (find_wmax); non-negative
// doubles order as their bit patterns
template <typename real>
__global__ void k_wmax(Geo G, Rng R, const real* __restrict__ w, unsigned long long* out)
{
    const int k = R.ks + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = R.js + blockIdx.y;
    const int i = R.is + blockIdx.z;
    double m = 0.0;
    if (k <= R.ke) {
        const double x = (double)w[(long)i * G.sx + (long)j * G.sy + k];
        m = (x > m) ? x : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double y = __shfl_xor_sync(0xffffffffu, m, o);
        m = (y > m) ? y : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// find_max, pass 1: max |x| of each field over the padded box (NaN never
// wins, as fabs(max) <= NaN is false); also the first linear index at which
// c_old, c_new or c's explicit term is NaN
template <typename real>
__global__ void k_absmax(Geo G, const real* __restrict__ f0, const real* __restrict__ f1,
                         const real* __restrict__ f2, const real* __restrict__ f3, const real* __restrict__ ca,
                         const real* __restrict__ cb, const real* __restrict__ cc, unsigned long long* out)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long n = (long)G.NX * G.NY * G.NZ;
    if (t >= n) return;
    const int i = (int)(t / ((long)G.NY * G.NZ));
    const int r = (int)(t % ((long)G.NY * G.NZ));
    const long id = (long)i * G.sx + (long)(r / G.NZ) * G.sy + (r % G.NZ);
    const real* fs[4] = {f0, f1, f2, f3};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double a = fabs((double)fs[q][id]);
        if (!isnan(a)) atomicMax(&out[q], (unsigned long long)__double_as_longlong(a));
    }
    if (isnan((double)ca[id]) || isnan((double)cb[id]) || isnan((double)cc[id]))
        atomicMin(&out[8], (unsigned long long)t);
}

// pass 2: the last linear index (i-j-k order) whose |x| equals the maximum
template <typename real>
__global__ void k_absmax_loc(Geo G, const real* __restrict__ f0, const real* __restrict__ f1,
                             const real* __restrict__ f2, const real* __restrict__ f3,
                             unsigned long long* out)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long n = (long)G.NX * G.NY * G.NZ;
    if (t >= n) return;
    const int i = (int)(t / ((long)G.NY * G.NZ));
    const int r = (int)(t % ((long)G.NY * G.NZ));
    const long id = (long)i * G.sx + (long)(r / G.NZ) * G.sy + (r % G.NZ);
    const real* fs[4] = {f0, f1, f2, f3};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double a = fabs((double)fs[q][id]);
        if (a == __longlong_as_double((long long)out[q])) atomicMax(&out[4 + q], (unsigned long long)t);
    }
}

// ---- host helpers --------------------------------------------------------------

std::string in_dir(const char* dir, const char* name)
{
    if (!dir || !*dir) return std::string(name);
    std::string s(dir);
    if (s.back() != '/') s += '/';
    return s + name;
}

// a device scratch buffer and a pinned host buffer of `bytes`, owned by the
// caller's scope
struct IoBufs {
    void* d = nullptr;
    void* h = nullptr;
    bool ok = false;
    explicit IoBufs(size_t bytes)
    {
        ok = cudaMalloc(&d, bytes > 0 ? bytes : 16) == cudaSuccess &&
             cudaMallocHost(&h, bytes > 0 ? bytes : 16) == cudaSuccess;
    }
    ~IoBufs()
    {
        if (d) cudaFree(d);
        if (h) cudaFreeHost(h);
    }
};

template <typename real>
MidPtrs<real> mid_ptrs(pllgpu_ctx* ctx, bool for_write)
{
    // midfield's order, pllcart3d.c:3160-3173
    static const int ids[NMID] = {PLLGPU_C_OLD,  PLLGPU_C_HNM1, PLLGPU_U_OLD, PLLGPU_U_NEW, PLLGPU_U_HNM1,
                                  PLLGPU_U_PG,   PLLGPU_V_OLD,  PLLGPU_V_NEW, PLLGPU_V_HNM1, PLLGPU_V_PG,
                                  PLLGPU_W_OLD,  PLLGPU_W_NEW,  PLLGPU_W_HNM1, PLLGPU_W_PG};
    MidPtrs<real> P{};
    for (int f = 0; f < NMID; ++f) P.f[f] = (real*)field_ptr(ctx, ids[f], for_write);
    return P;
}

template <typename real>
int write_mid_t(pllgpu_ctx* ctx, FILE* fp)
{
    const Geo& G = ctx->G;
    MidPtrs<real> P = mid_ptrs<real>(ctx, false);
    for (int f = 0; f < NMID; ++f)
        if (!P.f[f]) return fail(ctx, PLLGPU_ECUDA);
    const int chunk = 16;   // planes per copy
    const size_t per_plane = (size_t)G.NY * NMID * G.NZ;
    IoBufs B(sizeof(double) * per_plane * chunk);
    if (!B.ok) return fail(ctx, PLLGPU_ECUDA);
    for (int ia = 0; ia < G.NX; ia += chunk) {
        const int np = std::min(chunk, G.NX - ia);
        k_pack_mid<real><<<dim3((G.NZ + 127) / 128, G.NY, np), 128, 0, ctx->st>>>(G, P, ia, (double*)B.d);
        CK(cudaMemcpyAsync(B.h, B.d, sizeof(double) * per_plane * np, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (fwrite(B.h, sizeof(double), per_plane * np, fp) != per_plane * np) return fail(ctx, PLLGPU_EINVAL);
    }
    return PLLGPU_OK;
}

template <typename real>
int read_mid_t(pllgpu_ctx* ctx, FILE* fp)
{
    const Geo& G = ctx->G;
    MidPtrs<real> P = mid_ptrs<real>(ctx, true);
    for (int f = 0; f < NMID; ++f)
        if (!P.f[f]) return fail(ctx, PLLGPU_ECUDA);
    const int chunk = 16;
    const size_t per_plane = (size_t)G.NY * NMID * G.NZ;
    IoBufs B(sizeof(double) * per_plane * chunk);
    if (!B.ok) return fail(ctx, PLLGPU_ECUDA);
    for (int ia = 0; ia < G.NX; ia += chunk) {
        const int np = std::min(chunk, G.NX - ia);
        if (fread(B.h, sizeof(double), per_plane * np, fp) != per_plane * np) return fail(ctx, PLLGPU_EINVAL);
        CK(cudaMemcpyAsync(B.d, B.h, sizeof(double) * per_plane * np, cudaMemcpyHostToDevice, ctx->st));
        k_unpack_mid<real><<<dim3((G.NZ + 127) / 128, G.NY, np), 128, 0, ctx->st>>>(G, P, ia, (const double*)B.d);
        CK(cudaStreamSynchronize(ctx->st));
    }
    return PLLGPU_OK;
}

// even coordinates in [lo, hi]: first one and count
void evens(int lo, int hi, int& first, int& count)
{
    first = (lo % 2 == 0) ? lo : lo + 1;
    count = first > hi ? 0 : (hi - first) / 2 + 1;
}

template <typename real>
int snapshot_t(pllgpu_ctx* ctx, FILE* fp, int subsample)
{
    const Geo& G = ctx->G;
    const Rng& R = ctx->Rg;
    const real* u = (const real*)field_ptr(ctx, PLLGPU_U_NEW, false);
    const real* v = (const real*)field_ptr(ctx, PLLGPU_V_NEW, false);
    const real* w = (const real*)field_ptr(ctx, PLLGPU_W_NEW, false);
    const real* c = (const real*)field_ptr(ctx, PLLGPU_C_NEW, false);
    if (!u || !v || !w || !c) return fail(ctx, PLLGPU_ECUDA);
    int i0 = R.is, j0 = R.js, k0 = R.ks, st = 1;
    int ni = R.ie - R.is + 1, nj = R.je - R.js + 1, nk = R.ke - R.ks + 1;
    if (subsample) {
        st = 2;
        evens(R.is, R.ie, i0, ni);
        evens(R.js, R.je, j0, nj);
        evens(R.ks, R.ke, k0, nk);
    }
    const long total = (long)ni * nj * nk;
    IoBufs B(sizeof(float) * 4 * (size_t)total);
    if (!B.ok) return fail(ctx, PLLGPU_ECUDA);
    if (total > 0) {
        k_pack_caf<real><<<(unsigned)((total + 255) / 256), 256, 0, ctx->st>>>(G, u, v, w, c, i0, j0, k0, st, ni,
                                                                                nj, nk, (float*)B.d);
        CK(cudaMemcpyAsync(B.h, B.d, sizeof(float) * 4 * total, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (fwrite(B.h, sizeof(float), 4 * (size_t)total, fp) != 4 * (size_t)total) return fail(ctx, PLLGPU_EINVAL);
    }
    return PLLGPU_OK;
}

template <typename real>
int cavg_t(pllgpu_ctx* ctx, double tval, const char* dir)
{
    const Geo& G = ctx->G;
    const Rng& R = ctx->Rg;
    const real* c = (const real*)field_ptr(ctx, PLLGPU_C_NEW, false);
    if (!c) return fail(ctx, PLLGPU_ECUDA);
    const int ni = R.ie - R.is + 1, nj = R.je - R.js + 1, nk = R.ke - R.ks + 1;
    const size_t ny_n = (size_t)ni * nk, nz_n = (size_t)ni * nj;
    IoBufs B(sizeof(float) * (ny_n + nz_n + ni));
    if (!B.ok) return fail(ctx, PLLGPU_ECUDA);
    float* d = (float*)B.d;
    k_cavg_y<real><<<dim3((nk + 127) / 128, ni), 128, 0, ctx->st>>>(G, R, c, d);
    k_cavg_z<real><<<dim3((nj + 127) / 128, ni), 128, 0, ctx->st>>>(G, R, c, d + ny_n);
    k_cavg_yz<real><<<(ni + 127) / 128, 128, 0, ctx->st>>>(G, R, c, d + ny_n + nz_n);
    CK(cudaMemcpyAsync(B.h, B.d, sizeof(float) * (ny_n + nz_n + ni), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    const float* h = (const float*)B.h;
    FILE* fp = fopen(in_dir(dir, "cavgy.bin").c_str(), "ab");
    if (!fp) return fail(ctx, PLLGPU_EINVAL);
    fwrite(h, sizeof(float), ny_n, fp);
    fclose(fp);
    fp = fopen(in_dir(dir, "cavgz.bin").c_str(), "ab");
    if (!fp) return fail(ctx, PLLGPU_EINVAL);
    fwrite(h + ny_n, sizeof(float), nz_n, fp);
    fclose(fp);
    // cavgyz.bin: the time as float, then the yz averages (L3712-3726)
    fp = fopen(in_dir(dir, "cavgyz.bin").c_str(), "ab");
    if (!fp) return fail(ctx, PLLGPU_EINVAL);
    const float t = (float)tval;
    fwrite(&t, sizeof(float), 1, fp);
    fwrite(h + ny_n + nz_n, sizeof(float), ni, fp);
    fclose(fp);
    return PLLGPU_OK;
}

template <typename real>
int wmax_t(pllgpu_ctx* ctx, double* wmax)
{
    const Geo& G = ctx->G;
    const Rng& R = ctx->Rg;
    const real* w = (const real*)field_ptr(ctx, PLLGPU_W_NEW, false);
    if (!w) return fail(ctx, PLLGPU_ECUDA);
    IoBufs B(sizeof(unsigned long long));
    if (!B.ok) return fail(ctx, PLLGPU_ECUDA);
    CK(cudaMemsetAsync(B.d, 0, sizeof(unsigned long long), ctx->st));
    const int nk = R.ke - R.ks + 1, nj = R.je - R.js + 1, ni = R.ie - R.is + 1;
    k_wmax<real><<<dim3((nk + 31) / 32, nj, ni), 32, 0, ctx->st>>>(G, R, w, (unsigned long long*)B.d);
    CK(cudaMemcpyAsync(B.h, B.d, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    unsigned long long bits = *(unsigned long long*)B.h;
    std::memcpy(wmax, &bits, sizeof(double));
    return PLLGPU_OK;
}

template <typename real>
int findmax_t(pllgpu_ctx* ctx, double* val, int* loc, long* nan_at)
{
    const Geo& G = ctx->G;
    const real* f[4] = {(const real*)field_ptr(ctx, PLLGPU_U_NEW, false),
                        (const real*)field_ptr(ctx, PLLGPU_V_NEW, false),
                        (const real*)field_ptr(ctx, PLLGPU_W_NEW, false),
                        (const real*)field_ptr(ctx, PLLGPU_C_NEW, false)};
    const real* ca = (const real*)field_ptr(ctx, PLLGPU_C_OLD, false);
    const real* cb = f[3];
    const real* ch = (const real*)field_ptr(ctx, PLLGPU_C_HN, false);
    for (int q = 0; q < 4; ++q)
        if (!f[q]) return fail(ctx, PLLGPU_ECUDA);
    if (!ca || !ch) return fail(ctx, PLLGPU_ECUDA);
    IoBufs B(sizeof(unsigned long long) * 9);
    if (!B.ok) return fail(ctx, PLLGPU_ECUDA);
    unsigned long long init[9] = {0, 0, 0, 0, 0, 0, 0, 0, ~0ull};
    CK(cudaMemcpyAsync(B.d, init, sizeof(init), cudaMemcpyHostToDevice, ctx->st));
    const long n = (long)G.NX * G.NY * G.NZ;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    unsigned long long* d = (unsigned long long*)B.d;
    k_absmax<real><<<blocks, 256, 0, ctx->st>>>(G, f[0], f[1], f[2], f[3], ca, cb, ch, d);
    k_absmax_loc<real><<<blocks, 256, 0, ctx->st>>>(G, f[0], f[1], f[2], f[3], d);
    CK(cudaMemcpyAsync(B.h, B.d, sizeof(init), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    const unsigned long long* h = (const unsigned long long*)B.h;
    for (int q = 0; q < 4; ++q) {
        const long t = (long)h[4 + q];
        const int i = (int)(t / ((long)G.NY * G.NZ)), r = (int)(t % ((long)G.NY * G.NZ));
        loc[3 * q] = i;
        loc[3 * q + 1] = r / G.NZ;
        loc[3 * q + 2] = r % G.NZ;
        // the signed value at that index
        const real* p = (const real*)f[q] + (long)i * G.sx + (long)(r / G.NZ) * G.sy + (r % G.NZ);
        real v;
        CK(cudaMemcpy(&v, p, sizeof(real), cudaMemcpyDeviceToHost));
        val[q] = (double)v;
        // no finite |x| above 0 anywhere: the reference keeps max = 0 and
        // takes the last index whose |x| is 0 (the same rule)
    }
    *nan_at = h[8] == ~0ull ? -1 : (long)h[8];
    return PLLGPU_OK;
}

}  // namespace
}  // namespace pll

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int pllgpu_pack_cells(pllgpu_ctx* ctx, float* d_cells)
{
    if (!ctx || !d_cells || ((uintptr_t)d_cells & 15)) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    const Rng& R = ctx->Rg;
    const void* f[4] = {field_ptr(ctx, PLLGPU_U_NEW, false), field_ptr(ctx, PLLGPU_V_NEW, false),
                        field_ptr(ctx, PLLGPU_W_NEW, false), field_ptr(ctx, PLLGPU_C_NEW, false)};
    if (!f[0] || !f[1] || !f[2] || !f[3]) return fail(ctx, PLLGPU_ECUDA);
    const int ni = R.ie - R.is + 1, nj = R.je - R.js + 1, nk = R.ke - R.ks + 1;
    const long total = (long)ni * nj * nk;
    const unsigned blocks = (unsigned)((total + 255) / 256);
    if (ctx->mixed)
        k_pack_caf<float><<<blocks, 256, 0, ctx->st>>>(ctx->G, (const float*)f[0], (const float*)f[1],
                                                       (const float*)f[2], (const float*)f[3], R.is, R.js, R.ks, 1,
                                                       ni, nj, nk, d_cells);
    else
        k_pack_caf<double><<<blocks, 256, 0, ctx->st>>>(ctx->G, (const double*)f[0], (const double*)f[1],
                                                        (const double*)f[2], (const double*)f[3], R.is, R.js, R.ks, 1,
                                                        ni, nj, nk, d_cells);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

int pllgpu_unpack_cells(pllgpu_ctx* ctx, const float* d_cells)
{
    if (!ctx || !d_cells || ((uintptr_t)d_cells & 15)) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    void* f[4] = {field_ptr(ctx, PLLGPU_C_NEW, true), field_ptr(ctx, PLLGPU_U_NEW, true),
                  field_ptr(ctx, PLLGPU_V_NEW, true), field_ptr(ctx, PLLGPU_W_NEW, true)};
    if (!f[0] || !f[1] || !f[2] || !f[3]) return fail(ctx, PLLGPU_ECUDA);
    const Rng& R = ctx->Rg;
    const dim3 grid((unsigned)((R.ke - R.ks + 1 + 127) / 128), R.je - R.js + 1, R.ie - R.is + 1);
    if (ctx->mixed)
        k_unpack_cells<float><<<grid, 128, 0, ctx->st>>>(ctx->G, R, (const float4*)d_cells, (float*)f[0],
                                                         (float*)f[1], (float*)f[2], (float*)f[3]);
    else
        k_unpack_cells<double><<<grid, 128, 0, ctx->st>>>(ctx->G, R, (const float4*)d_cells, (double*)f[0],
                                                          (double*)f[1], (double*)f[2], (double*)f[3]);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

int pllgpu_write_snapshot_ex(pllgpu_ctx* ctx, int fileno, int rank, const char* dir, int subsample)
{
    if (!ctx || fileno < 0 || fileno > 9999 || rank < 0 || rank > 999) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    const Geo& G = ctx->G;
    if (subsample < 0) subsample = ((double)G.nx * G.ny * G.nz > 2e7) ? 1 : 0;   // L3079
    char name[32];
    snprintf(name, sizeof(name), "caf%04dR%03d.bin", fileno, rank);
    FILE* fp = fopen(in_dir(dir, name).c_str(), "wb");
    if (!fp) return fail(ctx, PLLGPU_EINVAL);
    const int e = ctx->mixed ? snapshot_t<float>(ctx, fp, subsample) : snapshot_t<double>(ctx, fp, subsample);
    fclose(fp);
    return e;
}

int pllgpu_write_snapshot(pllgpu_ctx* ctx, int fileno, const char* dir)
{
    return pllgpu_write_snapshot_ex(ctx, fileno, 0, dir, -1);
}

int pllgpu_write_restart(pllgpu_ctx* ctx, int tstep, int fileno, double tval, double outtime, double outmid,
                         double cavgtime, const char* dir)
{
    if (!ctx) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    FILE* fp = fopen(in_dir(dir, "middata").c_str(), "w");
    if (!fp) return fail(ctx, PLLGPU_EINVAL);
    fprintf(fp, "%d\n", tstep);
    fprintf(fp, "%d\n", fileno);
    fprintf(fp, "%lf\n", tval);
    fprintf(fp, "%lf\n", outtime);
    fprintf(fp, "%lf\n", outmid);
    fprintf(fp, "%lf\n", cavgtime);
    fclose(fp);
    fp = fopen(in_dir(dir, "midfield000.bin").c_str(), "wb");
    if (!fp) return fail(ctx, PLLGPU_EINVAL);
    const int e = ctx->mixed ? write_mid_t<float>(ctx, fp) : write_mid_t<double>(ctx, fp);
    fclose(fp);
    return e;
}

int pllgpu_read_restart(pllgpu_ctx* ctx, const char* dir, int* tstep, int* fileno, double* tval, double* outtime)
{
    if (!ctx || !tstep || !fileno || !tval || !outtime) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    FILE* fp = fopen(in_dir(dir, "middata").c_str(), "r");
    if (!fp) return fail(ctx, PLLGPU_EINVAL);
    const int got = fscanf(fp, "%d\n", tstep) + fscanf(fp, "%d\n", fileno) + fscanf(fp, "%lf\n", tval) +
                    fscanf(fp, "%lf\n", outtime);
    fclose(fp);
    if (got != 4) return fail(ctx, PLLGPU_EINVAL);
    if (int e = materialize(ctx)) return e;
    fp = fopen(in_dir(dir, "midfield000.bin").c_str(), "rb");
    if (!fp) return fail(ctx, PLLGPU_EINVAL);
    const int e = ctx->mixed ? read_mid_t<float>(ctx, fp) : read_mid_t<double>(ctx, fp);
    fclose(fp);
    return e;
}

int pllgpu_conc_average(pllgpu_ctx* ctx, double tval, const char* dir)
{
    if (!ctx) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    return ctx->mixed ? cavg_t<float>(ctx, tval, dir) : cavg_t<double>(ctx, tval, dir);
}

int pllgpu_find_wmax(pllgpu_ctx* ctx, double tval, const char* dir, double* wmax_out)
{
    if (!ctx) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    double wmax = 0;
    int e = ctx->mixed ? wmax_t<float>(ctx, &wmax) : wmax_t<double>(ctx, &wmax);
    if (e) return e;
    if (wmax_out) *wmax_out = wmax;
    if (dir) {
        FILE* fp = fopen(in_dir(dir, "wmax.bin").c_str(), "ab");
        if (!fp) return fail(ctx, PLLGPU_EINVAL);
        const float data[2] = {(float)wmax, (float)tval};
        fwrite(data, sizeof(float), 2, fp);
        fclose(fp);
    }
    return PLLGPU_OK;
}

int pllgpu_find_max(pllgpu_ctx* ctx, const char* dir, double* maxval, int* maxloc)
{
    if (!ctx) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    double val[4];
    int loc[12];
    long nan_at = -1;
    int e = ctx->mixed ? findmax_t<float>(ctx, val, loc, &nan_at) : findmax_t<double>(ctx, val, loc, &nan_at);
    if (e) return e;
    if (maxval) std::memcpy(maxval, val, sizeof(val));
    if (maxloc) std::memcpy(maxloc, loc, sizeof(loc));
    const Geo& G = ctx->G;
    if (nan_at >= 0) {
        // the first NaN in i-j-k order, named as the reference does
        // (a: c->old, b: c->new, c: c->explicit_n), L3567-3587
        const int i = (int)(nan_at / ((long)G.NY * G.NZ)), r = (int)(nan_at % ((long)G.NY * G.NZ));
        const int j = r / G.NZ, k = r % G.NZ;
        const long id = (long)i * G.sx + (long)j * G.sy + k;
        const int fid[3] = {PLLGPU_C_OLD, PLLGPU_C_NEW, PLLGPU_C_HN};
        const char tag[3] = {'a', 'b', 'c'};
        char which = 'a';
        for (int q = 0; q < 3; ++q) {
            double x;
            if (ctx->mixed) {
                float v;
                CK(cudaMemcpy(&v, (const float*)field_ptr(ctx, fid[q], false) + id, sizeof(float),
                              cudaMemcpyDeviceToHost));
                x = v;
            } else {
                CK(cudaMemcpy(&x, (const double*)field_ptr(ctx, fid[q], false) + id, sizeof(double),
                              cudaMemcpyDeviceToHost));
            }
            if (std::isnan(x)) {
                which = tag[q];
                break;
            }
        }
        if (dir) {
            FILE* fp = fopen(in_dir(dir, "Outscreen").c_str(), "a");
            if (fp) {
                fprintf(fp, "nan in %c %d %d %d \n", which, i, j, k);
                fclose(fp);
            }
        }
        return fail(ctx, PLLGPU_ENAN);
    }
    if (dir) {
        FILE* fp = fopen(in_dir(dir, "Outscreen").c_str(), "a");
        if (!fp) return fail(ctx, PLLGPU_EINVAL);
        fprintf(fp, "max\n");
        fprintf(fp, "  %2d %2d %2d %lf\n  %2d %2d %2d %lf\n  %2d %2d %2d %lf\n  %2d %2d %2d %lf\n\n", loc[0], loc[1],
                loc[2], val[0], loc[3], loc[4], loc[5], val[1], loc[6], loc[7], loc[8], val[2], loc[9], loc[10],
                loc[11], val[3]);
        fclose(fp);
    }
    return PLLGPU_OK;
}

}  // extern "C"
