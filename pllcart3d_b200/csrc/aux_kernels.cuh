// Viscosity, reductions, projection and ghost-fill kernels of the step.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "step_kernels.cuh"

namespace pll {
// internal linkage: each translation unit (and so each precision form with
// its own contraction flags) owns its instantiations
namespace {

// nmvp coefficient slots in the device scalar array
enum { S_MUM = 8, S_PSI0 = 9, S_PSI1 = 10, S_NMVA = 11 };

template <typename real>
__device__ __forceinline__ real visc_law(real cavg, const Consts& K, int nmvp,
                                         const double* __restrict__ scal)
{
    if (!nmvp) {
        // the precision form: the fast exponential (ex2-based, a few ulp for
        // the |M (c - Vnorm)| <= ~3 of these runs), FP32-level like its state
        if (sizeof(real) == 4) return (real)__expf((float)((real)K.M * (cavg - (real)K.Vnorm)));
        return (real)exp((double)((real)K.M * (cavg - (real)K.Vnorm)));
    }
    // calculate_viscosity_nmvp, pllcart3d.c:906-909
    const double a = scal[S_NMVA], psi0 = scal[S_PSI0], psi1 = scal[S_PSI1];
    double eta = ((1 + a) * (double)cavg) / (1 + a * (double)cavg);
    double psi = psi1 * (1 - eta) + psi0 * eta;
    return (real)(scal[S_MUM] * sin(psi));
}

// planes of i one k_viscosity thread walks
constexpr int VISC_NI = 4;

// calculate_viscosity (pllcart3d.c:843-886): mu at cell centres on the box
// padded by one cell, and on the xy / xz / yz edge families.  One thread per
// (j,k) of j in [0, NY-1], k in [0, NZ-1], walking VISC_NI planes of i in
// [is-1, ie+1]; the c values of plane i-1 that the xy and xz edges average
// come from the previous plane's registers.  Every point read lies inside the
// padded box's allocation (i >= is-1 >= 2), whether or not its value is used.
template <typename real>
__device__ __forceinline__ void k_viscosity_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, int nmvp,
                                                   const real* __restrict__ cn, real* __restrict__ mc,
                                                   real* __restrict__ mxy, real* __restrict__ mxz,
                                                   real* __restrict__ myz, const double* __restrict__ scal)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (k >= G.NZ || j >= G.NY) return;
    const int sx = (int)G.sx, sy = (int)G.sy;
    const int i0 = R.is - 1 + blockIdx.z * VISC_NI;
    const bool jxy = (j >= R.js) & (j <= R.je + 1), jin = (j >= R.js) & (j <= R.je);
    const bool kin = (k >= R.ks) & (k <= R.ke), kxz = (k >= R.ks) & (k <= R.ke + 1);
    const real q = (real)0.25;
    int id = i0 * sx + j * sy + k;
    // c at (i-1, j, k), (i-1, j-1, k), (i-1, j, k-1)
    real p0 = cn[id - sx], py = cn[id - sx - sy], pz = cn[id - sx - 1];
#pragma unroll
    for (int t = 0; t < VISC_NI; ++t, id += sx) {
        const int i = i0 + t;
        if (i > R.ie + 1) break;
        const real c0 = cn[id], cy = cn[id - sy], cz = cn[id - 1], cyz = cn[id - sy - 1];
        mc[id] = visc_law<real>(c0, K, nmvp, scal);
        const bool in_i = (i >= R.is), in_i2 = (i <= R.ie);
        if (in_i & jxy & kin) mxy[id] = visc_law<real>(q * (py + cy + p0 + c0), K, nmvp, scal);
        if (in_i & jin & kxz) mxz[id] = visc_law<real>(q * (pz + cz + p0 + c0), K, nmvp, scal);
        if (in_i & in_i2 & jxy & kxz) myz[id] = visc_law<real>(q * (cyz + cz + cy + c0), K, nmvp, scal);
        p0 = c0;
        py = cy;
        pz = cz;
    }
}
template <typename real>
__global__ void __launch_bounds__(128) k_viscosity(Geo G, Rng R, Consts K, int nmvp,
                                                   const real* __restrict__ cn, real* __restrict__ mc,
                                                   real* __restrict__ mxy, real* __restrict__ mxz,
                                                   real* __restrict__ myz, const double* __restrict__ scal)
{
    k_viscosity_run<real>(blockIdx, gridDim, G, R, K, nmvp, cn, mc, mxy, mxz, myz, scal);
}
template <typename real>
struct k_viscosity_b {
    static constexpr auto run = &k_viscosity_run<real>;
    static constexpr int maxt = 128, minb = 0;
};

// The exponential law on cell pairs (k, k+32): the precision form with
// packed FP32x2 arithmetic (the averages and exponents; __expf per value),
// the FP64 forms with FP64 pairs and exp(); walking
// VISC_NI planes as k_viscosity.  A second cell past NZ reads the slack past
// the array and stores nothing.  Grid: x over k in tiles of 64.
template <typename real>
__device__ __forceinline__ void k_viscosity2_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, const real* __restrict__ cn,
                                                    real* __restrict__ mc, real* __restrict__ mxy,
                                                    real* __restrict__ mxz, real* __restrict__ myz)
{
    using T2 = typename PairOf<real>::type;
    const int k = blockIdx.x * (2 * EP_DK) + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (k >= G.NZ || j >= G.NY) return;
    const int kb = k + EP_DK;
    const bool live_b = kb < G.NZ;
    const long sx = G.sx, sy = G.sy;
    const int i0 = R.is - 1 + blockIdx.z * VISC_NI;
    const bool jxy = (j >= R.js) & (j <= R.je + 1), jin = (j >= R.js) & (j <= R.je);
    const bool kin_a = (k >= R.ks) & (k <= R.ke), kxz_a = (k >= R.ks) & (k <= R.ke + 1);
    const bool kin_b = live_b & (kb <= R.ke), kxz_b = live_b & (kb <= R.ke + 1);
    const T2 q = S2((real)0.25), M = S2((real)K.M), Vn = S2((real)K.Vnorm);
    auto law = [&](T2 c) {
        const T2 t = M * (c - Vn);
        if constexpr (sizeof(real) == 4) return mk2(__expf(t.v.x), __expf(t.v.y));
        else return mk2(exp(t.v.x), exp(t.v.y));
    };
    long id = (long)i0 * sx + (long)j * sy + k;
    T2 p0 = ld2(cn, id - sx), py = ld2(cn, id - sx - sy), pz = ld2(cn, id - sx - 1);
#pragma unroll
    for (int t = 0; t < VISC_NI; ++t, id += sx) {
        const int i = i0 + t;
        if (i > R.ie + 1) break;
        const T2 c0 = ld2(cn, id), cy = ld2(cn, id - sy), cz = ld2(cn, id - 1), cyz = ld2(cn, id - sy - 1);
        const T2 vc = law(c0);
        mc[id] = vc.v.x;
        if (live_b) mc[id + EP_DK] = vc.v.y;
        const bool in_i = (i >= R.is), in_i2 = (i <= R.ie);
        if (in_i & jxy) {
            const T2 v = law(q * (py + cy + p0 + c0));
            if (kin_a) mxy[id] = v.v.x;
            if (kin_b) mxy[id + EP_DK] = v.v.y;
        }
        if (in_i & jin) {
            const T2 v = law(q * (pz + cz + p0 + c0));
            if (kxz_a) mxz[id] = v.v.x;
            if (kxz_b) mxz[id + EP_DK] = v.v.y;
        }
        if (in_i & in_i2 & jxy) {
            const T2 v = law(q * (cyz + cz + cy + c0));
            if (kxz_a) myz[id] = v.v.x;
            if (kxz_b) myz[id + EP_DK] = v.v.y;
        }
        p0 = c0;
        py = cy;
        pz = cz;
    }
}
template <typename real>
__global__ void __launch_bounds__(128) k_viscosity2(Geo G, Rng R, Consts K, const real* __restrict__ cn,
                                                    real* __restrict__ mc, real* __restrict__ mxy,
                                                    real* __restrict__ mxz, real* __restrict__ myz)
{
    k_viscosity2_run<real>(blockIdx, gridDim, G, R, K, cn, mc, mxy, mxz, myz);
}
template <typename real>
struct k_viscosity2_b {
    static constexpr auto run = &k_viscosity2_run<real>;
    static constexpr int maxt = 128, minb = 0;
};

// find_cfl (pllcart3d.c:3095-3118): max over interior cells of
// |u|/dx+|v|/dy+|w|/dz at cell centres, reduced exactly through the bit
// pattern of non-negative doubles; a NaN/Inf raises ST_NAN (the reference's
// NaN guard lives in find_max, pllcart3d.c:3568-3588)
template <typename real>
__device__ __forceinline__ void k_cfl_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, const real* __restrict__ u,
                                             const real* __restrict__ v, const real* __restrict__ w,
                                             double* scal, int* status)
{
    const int k = R.ks + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = R.js + blockIdx.y * blockDim.y + threadIdx.y;
    const int i = R.is + blockIdx.z;
    double m = 0.0;
    if (k <= R.ke && j <= R.je) {
        const long id = (long)i * G.sx + (long)j * G.sy + k;
        double uv = 0.5 * ((double)u[id] + (double)u[id + G.sx]);
        double vv = 0.5 * ((double)v[id] + (double)v[id + G.sy]);
        double wv = 0.5 * ((double)w[id] + (double)w[id + 1]);
#if PLL_FP64_EXACT
        double cfl = (fabs(uv) / K.hx) + (fabs(vv) / K.hy) + (fabs(wv) / K.hz);
#else
        // the FP64 forms: reciprocal spacings, the fusions written out
        double cfl = fma(fabs(wv), K.ihz, fma(fabs(vv), K.ihy, fabs(uv) * K.ihx));
#endif
        if (!isfinite(cfl)) atomicOr(status, (int)ST_NAN);
        else m = cfl;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double sm[8];
    const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
    const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    if (lane == 0) sm[warp] = m;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x * blockDim.y) >> 5;
        m = lane < nw ? sm[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0 && m > 0.0)
            atomicMax((unsigned long long*)(scal + S_CFLMAX), (unsigned long long)__double_as_longlong(m));
    }
}
template <typename real>
__global__ void __launch_bounds__(256) k_cfl(Geo G, Rng R, Consts K, const real* __restrict__ u,
                                             const real* __restrict__ v, const real* __restrict__ w,
                                             double* scal, int* status)
{
    k_cfl_run<real>(blockIdx, gridDim, G, R, K, u, v, w, scal, status);
}
template <typename real>
struct k_cfl_b {
    static constexpr auto run = &k_cfl_run<real>;
    static constexpr int maxt = 256, minb = 0;
};

// dt = min(CFLmax / max, Timestep), pllcart3d.c:159-160, 3115; clears the
// reduction slot for the next step
static __device__ __forceinline__ void k_dt_run(const uint3 blockIdx, const dim3 gridDim,
    Consts K, double* scal)
{
    double maxall = __longlong_as_double((long long)*(unsigned long long*)(scal + S_CFLMAX));
    double cfldt = K.CFLmax / maxall;
    double ts = scal[S_TIMESTEP];
    scal[S_CFLDT] = cfldt;
    scal[S_DT] = (cfldt < ts) ? cfldt : ts;
    *(unsigned long long*)(scal + S_CFLMAX) = 0ull;
}
static __global__ void k_dt(Consts K, double* scal)
{
    k_dt_run(blockIdx, gridDim, K, scal);
}
struct k_dt_b {
    static constexpr auto run = &k_dt_run;
    static constexpr int maxt = 0, minb = 0;
};

// inflow/outflow trapezoid fluxes of velo_correction (pllcart3d.c:2171-2223):
// per y row a sequential sum over z of 0.5*dz*(u_k+u_{k-1}) from k=ks+1,
// then a sequential sum over y of 0.5*dy*(q_{j-1}+q_j) from j=js+1 (wall
// half-cells excluded), in the reference's order.  One block.
template <typename real>
__device__ __forceinline__ void k_flux_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng Ru, Consts K, const real* __restrict__ u,
                                              double* scal)
{
    extern __shared__ double qk[];  // 2 * NY
    const int iin = Ru.is - 1, iout = Ru.ie + 1;
    const double hdz = 0.5 * K.hz, hdy = 0.5 * K.hy;
    for (int j = Ru.js + threadIdx.x; j <= Ru.je; j += blockDim.x) {
        double qi = 0.0, qo = 0.0;
        const long bi = (long)iin * G.sx + (long)j * G.sy, bo = (long)iout * G.sx + (long)j * G.sy;
        for (int k = Ru.ks + 1; k <= Ru.ke; ++k) {
            qi += hdz * ((double)u[bi + k] + (double)u[bi + k - 1]);
            qo += hdz * ((double)u[bo + k] + (double)u[bo + k - 1]);
        }
        qk[j] = qi;
        qk[G.NY + j] = qo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double qin = 0.0, qout = 0.0;
        for (int j = Ru.js + 1; j <= Ru.je; ++j) {
            qin += hdy * (qk[j - 1] + qk[j]);
            qout += hdy * (qk[G.NY + j - 1] + qk[G.NY + j]);
        }
        scal[S_QIN] = qin;
        scal[S_QOUT] = qout;
        scal[S_DEFICIT] = (qin - qout) / K.area;
    }
}
template <typename real>
__global__ void __launch_bounds__(512) k_flux(Geo G, Rng Ru, Consts K, const real* __restrict__ u,
                                              double* scal)
{
    k_flux_run<real>(blockIdx, gridDim, G, Ru, K, u, scal);
}
template <typename real>
struct k_flux_b {
    static constexpr auto run = &k_flux_run<real>;
    static constexpr int maxt = 512, minb = 0;
};

// The precision form's Poisson right-hand side (k_div_rhs mode 0) on cell
// pairs (k, k+32) with packed FP32x2 arithmetic, each thread walking
// DIV_NI planes with u at the next plane carried in registers.  A second
// cell past ke reads the slack past the arrays and stores nothing.
constexpr int DIV_NI = 4;

template <typename real>
__device__ __forceinline__ void k_div_rhs2_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, const real* __restrict__ u,
                                                  const real* __restrict__ v, const real* __restrict__ w,
                                                  real* __restrict__ rhs, const double* __restrict__ scal,
                                                  double alpha)
{
    using T2 = typename PairOf<real>::type;
    const int k = R.ks + blockIdx.x * (2 * EP_DK) + threadIdx.x;
    const int j = R.js + blockIdx.y * blockDim.y + threadIdx.y;
    if (k > R.ke || j > R.je) return;
    const bool live_b = k + EP_DK <= R.ke;
    const int i0 = R.is + blockIdx.z * DIV_NI;
    const long sx = G.sx, sy = G.sy;
    const T2 ihx = S2((real)K.ihx), ihy = S2((real)K.ihy), ihz = S2((real)K.ihz);
    const T2 fac = S2((real)(K.Re / (scal[S_DT] * alpha)));
    const long nj = R.je - R.js + 1, nkk = R.ke - R.ks + 1;
    long id = (long)i0 * sx + (long)j * sy + k;
    T2 u0 = ld2(u, id);
#pragma unroll
    for (int t = 0; t < DIV_NI; ++t, id += sx) {
        const int i = i0 + t;
        if (i > R.ie) break;
        const T2 u1 = ld2(u, id + sx);
        const T2 dvx = (u1 - u0) * ihx;
        const T2 dvy = (ld2(v, id + sy) - ld2(v, id)) * ihy;
        const T2 dvz = (ld2(w, id + 1) - ld2(w, id)) * ihz;
        const T2 r = fac * (dvx + dvy + dvz);
        const long c = ((long)(i - R.is) * nj + (j - R.js)) * nkk + (k - R.ks);
        rhs[c] = r.v.x;
        if (live_b) rhs[c + EP_DK] = r.v.y;
        u0 = u1;
    }
}
template <typename real>
__global__ void __launch_bounds__(128) k_div_rhs2(Geo G, Rng R, Consts K, const real* __restrict__ u,
                                                  const real* __restrict__ v, const real* __restrict__ w,
                                                  real* __restrict__ rhs, const double* __restrict__ scal,
                                                  double alpha)
{
    k_div_rhs2_run<real>(blockIdx, gridDim, G, R, K, u, v, w, rhs, scal, alpha);
}
template <typename real>
struct k_div_rhs2_b {
    static constexpr auto run = &k_div_rhs2_run<real>;
    static constexpr int maxt = 128, minb = 0;
};

// The precision form's CFL scan: cell pairs (k, k+32), CFL_NI planes per
// thread, the per-cell speed sum in FP64 (the reciprocal spacings multiply:
// the precision form's dt may differ from the division's in the last bit)
// and a thread-local maximum before the warp and block reductions.  The
// maximum itself does not depend on the order.  A second cell past ke reads
// the slack past the arrays and is left out.
constexpr int CFL_NI = 8;

__device__ __forceinline__ void k_cfl2_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, const float* __restrict__ u,
                                              const float* __restrict__ v, const float* __restrict__ w, double* scal,
                                              int* status)
{
    const int k = R.ks + blockIdx.x * (2 * EP_DK) + threadIdx.x;
    const int j = R.js + blockIdx.y * blockDim.y + threadIdx.y;
    const int i0 = R.is + blockIdx.z * CFL_NI;
    double m = 0.0;
    bool bad = false;
    if (k <= R.ke && j <= R.je) {
        const bool live_b = k + EP_DK <= R.ke;
        const long sx = G.sx, sy = G.sy;
        long id = (long)i0 * sx + (long)j * sy + k;
        f2 u0 = ld2(u, id);
#pragma unroll
        for (int t = 0; t < CFL_NI; ++t, id += sx) {
            if (i0 + t > R.ie) break;
            const f2 u1 = ld2(u, id + sx), v0 = ld2(v, id), v1 = ld2(v, id + sy), w0 = ld2(w, id), w1 = ld2(w, id + 1);
            double ca = fabs(0.5 * ((double)u0.v.x + (double)u1.v.x)) * K.ihx +
                        fabs(0.5 * ((double)v0.v.x + (double)v1.v.x)) * K.ihy +
                        fabs(0.5 * ((double)w0.v.x + (double)w1.v.x)) * K.ihz;
            double cb = fabs(0.5 * ((double)u0.v.y + (double)u1.v.y)) * K.ihx +
                        fabs(0.5 * ((double)v0.v.y + (double)v1.v.y)) * K.ihy +
                        fabs(0.5 * ((double)w0.v.y + (double)w1.v.y)) * K.ihz;
            if (!live_b) cb = 0.0;
            if (isfinite(ca)) m = fmax(m, ca);
            else bad = true;
            if (isfinite(cb)) m = fmax(m, cb);
            else bad = true;
            u0 = u1;
        }
    }
    if (bad) atomicOr(status, (int)ST_NAN);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double sm[8];
    const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
    const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    if (lane == 0) sm[warp] = m;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x * blockDim.y) >> 5;
        m = lane < nw ? sm[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0 && m > 0.0)
            atomicMax((unsigned long long*)(scal + S_CFLMAX), (unsigned long long)__double_as_longlong(m));
    }
}
__global__ void __launch_bounds__(256) k_cfl2(Geo G, Rng R, Consts K, const float* __restrict__ u,
                                              const float* __restrict__ v, const float* __restrict__ w, double* scal,
                                              int* status)
{
    k_cfl2_run(blockIdx, gridDim, G, R, K, u, v, w, scal, status);
}
struct k_cfl2_b {
    static constexpr auto run = &k_cfl2_run;
    static constexpr int maxt = 256, minb = 0;
};

// Last-block ticket: every block's results are written and fenced before it
// takes a ticket; the block that takes the last one reads them all and
// resets the counter for the next launch.
__device__ __forceinline__ bool last_block(unsigned* ticket)
{
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// The precision form's inflow/outflow fluxes: the trapezoid sums of k_flux
// in FP64, evaluated in parallel in a fixed order (every run gives the same
// bits): one warp per row of either plane, lane l summing the terms k =
// ks+1+l, ks+1+l+32, ... and a fixed shuffle tree; the last block forms the
// sum over y the same way from the row sums.  Blocks of 1024 threads.
__device__ __forceinline__ void k_flux3_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng Ru, Consts K, const float* __restrict__ u, double* red,
                                                unsigned* ticket, double* scal)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nyr = Ru.je - Ru.js + 1;
    const double hdz = 0.5 * K.hz, hdy = 0.5 * K.hy;
    auto tree = [&](double x) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        return x;
    };
    const int r = blockIdx.x * 32 + warp;   // row of plane r / nyr
    if (r < 2 * nyr) {
        const int plane = r / nyr, j = Ru.js + r % nyr;
        const long b = (long)(plane ? Ru.ie + 1 : Ru.is - 1) * G.sx + (long)j * G.sy;
        double q = 0.0;
        for (int k = Ru.ks + 1 + lane; k <= Ru.ke; k += 32) q += hdz * ((double)u[b + k] + (double)u[b + k - 1]);
        q = tree(q);
        if (lane == 0) red[plane * G.NY + j] = q;
    }
    if (!last_block(ticket)) return;
    if (warp == 0) {
        double qin = 0.0, qout = 0.0;
        for (int j = Ru.js + 1 + lane; j <= Ru.je; j += 32) {
            qin += hdy * (__ldcg(red + j - 1) + __ldcg(red + j));
            qout += hdy * (__ldcg(red + G.NY + j - 1) + __ldcg(red + G.NY + j));
        }
        qin = tree(qin);
        qout = tree(qout);
        if (lane == 0) {
            scal[S_QIN] = qin;
            scal[S_QOUT] = qout;
            scal[S_DEFICIT] = (qin - qout) / K.area;
            *ticket = 0u;
        }
    }
}
__global__ void __launch_bounds__(1024) k_flux3(Geo G, Rng Ru, Consts K, const float* __restrict__ u, double* red,
                                                unsigned* ticket, double* scal)
{
    k_flux3_run(blockIdx, gridDim, G, Ru, K, u, red, ticket, scal);
}
struct k_flux3_b {
    static constexpr auto run = &k_flux3_run;
    static constexpr int maxt = 1024, minb = 0;
};

// bulk_velo (pllcart3d.c:3381-3398): the signed value of the first (j-major,
// k-minor) entry of largest |u| on the face i = iend; 0 if all are 0.  Over
// BULK_BLOCKS blocks: each block reduces a strided share keeping the smallest
// index among equal values, the last block the block partials; the result
// does not depend on the order.
template <typename real>
__device__ __forceinline__ void k_bulk2_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, const real* __restrict__ u, double* red,
                                               unsigned* ticket, double* scal)
{
    const int nyz = (R.je - R.js + 1) * (R.ke - R.ks + 1), nk = R.ke - R.ks + 1;
    double best = 0.0;
    int bidx = 0x7fffffff;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nyz; t += gridDim.x * blockDim.x) {
        const int j = R.js + t / nk, k = R.ks + t % nk;
        const double a = fabs((double)u[(long)R.ie * G.sx + (long)j * G.sy + k]);
        if (a > best) { best = a; bidx = t; }
    }
    auto merge = [](double& b, int& i, double b2, int i2) {
        if (b2 > b || (b2 == b && i2 < i)) { b = b2; i = i2; }
    };
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double b2 = __shfl_xor_sync(0xffffffffu, best, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, bidx, o);
        merge(best, bidx, b2, i2);
    }
    __shared__ double sb[32];
    __shared__ int si[32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { sb[warp] = best; si[warp] = bidx; }
    __syncthreads();
    double* pv = red + 2L * G.NY;
    double* pi = pv + BULK_BLOCKS;
    if (warp == 0) {
        best = lane < (int)(blockDim.x >> 5) ? sb[lane] : 0.0;
        bidx = lane < (int)(blockDim.x >> 5) ? si[lane] : 0x7fffffff;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double b2 = __shfl_xor_sync(0xffffffffu, best, o);
            const int i2 = __shfl_xor_sync(0xffffffffu, bidx, o);
            merge(best, bidx, b2, i2);
        }
        if (lane == 0) { pv[blockIdx.x] = best; pi[blockIdx.x] = (double)bidx; }
    }
    if (!last_block(ticket)) return;
    if (warp == 0) {
        best = 0.0;
        bidx = 0x7fffffff;
        for (int b = lane; b < (int)gridDim.x; b += 32) merge(best, bidx, __ldcg(pv + b), (int)__ldcg(pi + b));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double b2 = __shfl_xor_sync(0xffffffffu, best, o);
            const int i2 = __shfl_xor_sync(0xffffffffu, bidx, o);
            merge(best, bidx, b2, i2);
        }
        if (lane == 0) {
            double vb = 0.0;
            if (best > 0.0) {
                const int j = R.js + bidx / nk, k = R.ks + bidx % nk;
                vb = (double)u[(long)R.ie * G.sx + (long)j * G.sy + k];
            }
            scal[S_VBULK] = vb;
            *ticket = 0u;
        }
    }
}
template <typename real>
__global__ void __launch_bounds__(1024) k_bulk2(Geo G, Rng R, const real* __restrict__ u, double* red,
                                               unsigned* ticket, double* scal)
{
    k_bulk2_run<real>(blockIdx, gridDim, G, R, u, red, ticket, scal);
}
template <typename real>
struct k_bulk2_b {
    static constexpr auto run = &k_bulk2_run<real>;
    static constexpr int maxt = 1024, minb = 0;
};

// divergence (pllcart3d.c:1983-1999) scaled by Re/(dt alpha)
// (phisolver_dct L2010-2024) into the compact [x][y][z] Poisson buffer.
// With `div_out` set, the unscaled divergence also goes to the padded field.
template <typename real>
__device__ __forceinline__ void k_div_rhs_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, const real* __restrict__ u,
                                                 const real* __restrict__ v, const real* __restrict__ w,
                                                 const real* __restrict__ div_in, real* __restrict__ div_out,
                                                 real* __restrict__ rhs, const double* __restrict__ scal,
                                                 double alpha, int mode)
{
    // mode 0: rhs from u,v,w ; 1: div_out from u,v,w ; 2: rhs from div_in
    const int k = R.ks + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = R.js + blockIdx.y * blockDim.y + threadIdx.y;
    const int i = R.is + blockIdx.z;
    if (k > R.ke || j > R.je) return;
    const long id = (long)i * G.sx + (long)j * G.sy + k;
    real d;
    if (mode == 2) {
        d = div_in[id];
    } else {
        real dvx = over_h<real>(u[id + G.sx] - u[id], K.hx, K.ihx, K.pow2);
        real dvy = over_h<real>(v[id + G.sy] - v[id], K.hy, K.ihy, K.pow2);
        real dvz = over_h<real>(w[id + 1] - w[id], K.hz, K.ihz, K.pow2);
        d = (dvx + dvy + dvz);
        if (mode == 1) {
            div_out[id] = d;
            return;
        }
    }
    const real fac = (real)(K.Re / (scal[S_DT] * alpha));
    const long c = ((long)(i - R.is) * (R.je - R.js + 1) + (j - R.js)) * (long)(R.ke - R.ks + 1) + (k - R.ks);
    rhs[c] = fac * d;
}
template <typename real>
__global__ void __launch_bounds__(128) k_div_rhs(Geo G, Rng R, Consts K, const real* __restrict__ u,
                                                 const real* __restrict__ v, const real* __restrict__ w,
                                                 const real* __restrict__ div_in, real* __restrict__ div_out,
                                                 real* __restrict__ rhs, const double* __restrict__ scal,
                                                 double alpha, int mode)
{
    k_div_rhs_run<real>(blockIdx, gridDim, G, R, K, u, v, w, div_in, div_out, rhs, scal, alpha, mode);
}
template <typename real>
struct k_div_rhs_b {
    static constexpr auto run = &k_div_rhs_run<real>;
    static constexpr int maxt = 128, minb = 0;
};

// x-direction tridiagonal of each (ky,kz) Poisson mode (phisolver_dct
// pllcart3d.c:2040-2091): a = c = 1/dx^2, b = -2/dx^2 + lam_y + lam_z,
// Neumann at the inlet, and at the outlet Neumann except for mode (0,0),
// whose right ghost holds phi = 0 (the pressure gauge); pll_tridiag's
// one-rank arithmetic.  One thread per mode; lines of stride ny*nz.  The
// mode coefficients are stored as T (the precision form keeps them in FP32)
// but the solve, the eigenvalue division and the zero mode are FP64, with
// c' and the eliminated rhs in FP64 scratch.
template <typename T>
__device__ __forceinline__ void k_poisson_x_run(const uint3 blockIdx, const dim3 gridDim,
    int nx, int ny, int nz, Consts K,
                                                   const double* __restrict__ lam_y,
                                                   const double* __restrict__ lam_z,
                                                   T* __restrict__ hat, double* __restrict__ cc,
                                                   double* __restrict__ rr, int kz_major = 0)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ny * nz) return;
    // modes stored [x][ky][kz] (kz_major 0) or [x][kz][ky] (kz_major 1)
    const int jy = kz_major ? t % ny : t / nz, kz = kz_major ? t / ny : t % nz;
    const long st = (long)ny * nz;
    const double a = K.dx2i, c = K.dx2i;
    const double bmid = -2.0 * K.dx2i + lam_y[jy] + lam_z[kz];
    const bool gauge = (jy == 0) && (kz == 0);
    // the loads of PF positions ahead are issued before the recurrence
    // consumes the current ones (the line is strided by ny*nz)
    constexpr int PF = 8;
    double cprev = 0, rprev = 0;
    T hv[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) hv[u] = u < nx ? hat[t + (long)u * st] : (T)0;
    for (int m0 = 0; m0 < nx; m0 += PF) {
        T hn[PF];
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int m = m0 + PF + u;
            hn[u] = m < nx ? hat[t + (long)m * st] : (T)0;
        }
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int m = m0 + u;
            if (m < nx) {
                const long id = t + (long)m * st;
                double lb = bmid, lr = (double)hv[u];
                if (m == 0) lb += a;
                if (m == nx - 1) {
                    if (gauge) lr -= c * 0.0;
                    else lb += c;
                }
                double cm, rm;   // the FP64 forms divide once (thomas_div)
                if (m == 0) {
                    lb = lb - 0.0 * a;
                    thomas_div<double>(c, (lr - 0.0 * a), lb, cm, rm);
                } else {
                    lb = (lb - cprev * a);
                    thomas_div<double>(c, (lr - rprev * a), lb, cm, rm);
                }
                cc[id] = cm;
                rr[id] = rm;
                cprev = cm;
                rprev = rm;
            }
        }
#pragma unroll
        for (int u = 0; u < PF; ++u) hv[u] = hn[u];
    }
    double xnext = rprev - cprev * 0.0;
    hat[t + (long)(nx - 1) * st] = (T)xnext;
    double rv[PF], cv[PF];
    int mtop = nx - 2;
#pragma unroll
    for (int u = 0; u < PF; ++u) {
        const int m = mtop - u;
        rv[u] = m >= 0 ? rr[t + (long)m * st] : 0.0;
        cv[u] = m >= 0 ? cc[t + (long)m * st] : 0.0;
    }
    for (; mtop >= 0; mtop -= PF) {
        double rn[PF], cn[PF];
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int m = mtop - PF - u;
            rn[u] = m >= 0 ? rr[t + (long)m * st] : 0.0;
            cn[u] = m >= 0 ? cc[t + (long)m * st] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int m = mtop - u;
            if (m >= 0) {
                const double x = rv[u] - cv[u] * xnext;
                hat[t + (long)m * st] = (T)x;
                xnext = x;
            }
        }
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            rv[u] = rn[u];
            cv[u] = cn[u];
        }
    }
}
template <typename T>
__global__ void __launch_bounds__(128) k_poisson_x(int nx, int ny, int nz, Consts K,
                                                   const double* __restrict__ lam_y,
                                                   const double* __restrict__ lam_z,
                                                   T* __restrict__ hat, double* __restrict__ cc,
                                                   double* __restrict__ rr, int kz_major = 0)
{
    k_poisson_x_run<T>(blockIdx, gridDim, nx, ny, nz, K, lam_y, lam_z, hat, cc, rr, kz_major);
}
template <typename T>
struct k_poisson_x_b {
    static constexpr auto run = &k_poisson_x_run<T>;
    static constexpr int maxt = 128, minb = 0;
};

// update_phi_ghosts (pllcart3d.c:2758-2807): Neumann copies on the six
// faces; FACE 0: z faces over (i,j), 1: y faces over (i,k), 2: x faces over
// (j,k)
template <int FACE, typename real>
__device__ __forceinline__ void k_phi_ghosts_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, real* __restrict__ p)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    const long sx = G.sx, sy = G.sy;
    if (FACE == 0) {
        const int j = R.js + a, i = R.is + b;
        if (j > R.je) return;
        const long base = (long)i * sx + (long)j * sy;
        p[base + R.ks - 1] = p[base + R.ks];
        p[base + R.ke + 1] = p[base + R.ke];
    } else if (FACE == 1) {
        const int k = R.ks + a, i = R.is + b;
        if (k > R.ke) return;
        const long base = (long)i * sx + k;
        p[base + (long)(R.js - 1) * sy] = p[base + (long)R.js * sy];
        p[base + (long)(R.je + 1) * sy] = p[base + (long)R.je * sy];
    } else {
        const int k = R.ks + a, j = R.js + b;
        if (k > R.ke) return;
        const long base = (long)j * sy + k;
        p[base + (long)(R.is - 1) * sx] = p[base + (long)R.is * sx];
        p[base + (long)(R.ie + 1) * sx] = p[base + (long)R.ie * sx];
    }
}
template <int FACE, typename real>
__global__ void k_phi_ghosts(Geo G, Rng R, real* __restrict__ p)
{
    k_phi_ghosts_run<FACE, real>(blockIdx, gridDim, G, R, p);
}
template <int FACE, typename real>
struct k_phi_ghosts_b {
    static constexpr auto run = &k_phi_ghosts_run<FACE, real>;
    static constexpr int maxt = 0, minb = 0;
};

// planes of i one k_project thread walks
constexpr int PROJECT_NI = 1;

// accumulated pressure gradient pold of component VAR at id advanced by
// grad(phi) along its axis and the viscous operator applied to that gradient
template <int VAR, typename real>
__device__ __forceinline__ real pg_update(const Consts& K, const Geo& G, const real* __restrict__ phi,
                                          const real* __restrict__ mc, const real* __restrict__ mxy,
                                          const real* __restrict__ mxz, const real* __restrict__ myz,
                                          int id, int sx, int sy, real fac, real pold)
{
    const int so = VAR == VU ? sx : VAR == VV ? sy : 1;
    const double h = VAR == VU ? K.hx : VAR == VV ? K.hy : K.hz;
    const double ih = VAR == VU ? K.ihx : VAR == VV ? K.ihy : K.ihz;
    auto gp = [&](int p) { return over_h<real>(phi[p] - phi[p - so], h, ih, K.pow2); };
    real a, b, c;
    const real g0 = gp(id);
    acoef<VAR, 0, real>(K, G, mc, mxy, mxz, myz, id, a, b, c);
    const real pxx = a * gp(id - sx) + b * g0 + c * gp(id + sx);
    acoef<VAR, 1, real>(K, G, mc, mxy, mxz, myz, id, a, b, c);
    const real pyy = a * gp(id - sy) + b * g0 + c * gp(id + sy);
    acoef<VAR, 2, real>(K, G, mc, mxy, mxz, myz, id, a, b, c);
    const real pzz = a * gp(id - 1) + b * g0 + c * gp(id + 1);
    return pold + g0 - fac * (pyy + pxx + pzz);
}

// velo_correction (pllcart3d.c:2133-2227), update_veloghost_points
// (L2810-2885) and pressure_gradient (L2964-3044) fused: one thread per
// (j,k) of j in [js, je], k in [ks, ke], walking PROJECT_NI planes of i in
// [is, ie+1].  Ghost copies are written by the thread that owns their source
// value, after its correction.  grad(phi) at neighbours is evaluated from phi
// directly (the reference's phi_x/phi_y/phi_z temporaries hold exactly these
// values).  Every pointer is a restrict-qualified parameter: the outputs
// (u, v, w, pg) are written only at points no thread of the launch reads
// (a thread's own u, v, w and ghosts outside the walked range), so the loads
// of both planes may all be in flight before the first store.
template <typename real>
__device__ __forceinline__ void k_project_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng Rg, Rng Ru, Rng Rv, Rng Rw, Consts K,
        real* __restrict__ u, real* __restrict__ v, real* __restrict__ w,
        real* __restrict__ pgu, real* __restrict__ pgv, real* __restrict__ pgw,
        const real* __restrict__ phi, const real* __restrict__ mc, const real* __restrict__ mxy,
        const real* __restrict__ mxz, const real* __restrict__ myz, const double* __restrict__ scal,
        double alpha, int do_correct, int do_ghosts, int do_pg)
{
    const int k = Rg.ks + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = Rg.js + blockIdx.y * blockDim.y + threadIdx.y;
    if (k > Rg.ke || j > Rg.je) return;
    const int sx = (int)G.sx, sy = (int)G.sy;
    const double dt = scal[S_DT];
    const real cfac = (real)(dt * alpha / K.Re);
    const real pfac = (real)(0.5 * dt * alpha);
#pragma unroll
    for (int t = 0; t < PROJECT_NI; ++t) {
        const int i = Rg.is + blockIdx.z * PROJECT_NI + t;
        if (i > Rg.ie + 1) break;
        const int id = i * sx + j * sy + k;
        const bool inu = (i >= Ru.is) & (i <= Ru.ie) & (j >= Ru.js) & (k >= Ru.ks);
        const bool inv = (i <= Rv.ie) & (j >= Rv.js) & (k >= Rv.ks);
        const bool inw = (i <= Rw.ie) & (j >= Rw.js) & (k >= Rw.ks);
        const bool ghost_i = (i <= Rg.ie);

        if (do_correct) {
            real uval = u[id], vval = 0, wval = 0;
            if (ghost_i) {
                vval = v[id];
                wval = w[id];
            }
            if (inv) {
                vval = vval - cfac * over_h<real>(phi[id] - phi[id - sy], K.hy, K.ihy, K.pow2);
                v[id] = vval;
            }
            if (inw) {
                wval = wval - cfac * over_h<real>(phi[id] - phi[id - 1], K.hz, K.ihz, K.pow2);
                w[id] = wval;
            }
            if (inu) {
                uval = uval - cfac * over_h<real>(phi[id] - phi[id - sx], K.hx, K.ihx, K.pow2);
                u[id] = uval;
            }
            if (i == Ru.ie + 1 && j >= Ru.js && k >= Ru.ks) u[id] = uval + (real)scal[S_DEFICIT];
            if (do_ghosts && ghost_i) {
                if (k == Rg.ks) { u[id - 1] = uval; v[id - 1] = vval; }
                if (k == Rg.ke) { u[id + 1] = uval; v[id + 1] = vval; }
                if (j == Rg.js) { u[id - sy] = -uval; w[id - sy] = -wval; }
                if (j == Rg.je) { u[id + sy] = -uval; w[id + sy] = -wval; }
                if (i == Rg.is) { v[id - sx] = -vval; w[id - sx] = -wval; }
            }
        } else if (do_ghosts && ghost_i) {
            const real uval = u[id], vval = v[id], wval = w[id];
            if (k == Rg.ks) { u[id - 1] = uval; v[id - 1] = vval; }
            if (k == Rg.ke) { u[id + 1] = uval; v[id + 1] = vval; }
            if (j == Rg.js) { u[id - sy] = -uval; w[id - sy] = -wval; }
            if (j == Rg.je) { u[id + sy] = -uval; w[id + sy] = -wval; }
            if (i == Rg.is) { v[id - sx] = -vval; w[id - sx] = -wval; }
        }

        if (do_pg) {
            if (inv) pgv[id] = pg_update<VV, real>(K, G, phi, mc, mxy, mxz, myz, id, sx, sy, pfac, pgv[id]);
            if (inu) pgu[id] = pg_update<VU, real>(K, G, phi, mc, mxy, mxz, myz, id, sx, sy, pfac, pgu[id]);
            if (inw) pgw[id] = pg_update<VW, real>(K, G, phi, mc, mxy, mxz, myz, id, sx, sy, pfac, pgw[id]);
        }
    }
}
template <typename real>
__global__ void __launch_bounds__(128) k_project(Geo G, Rng Rg, Rng Ru, Rng Rv, Rng Rw, Consts K,
        real* __restrict__ u, real* __restrict__ v, real* __restrict__ w,
        real* __restrict__ pgu, real* __restrict__ pgv, real* __restrict__ pgw,
        const real* __restrict__ phi, const real* __restrict__ mc, const real* __restrict__ mxy,
        const real* __restrict__ mxz, const real* __restrict__ myz, const double* __restrict__ scal,
        double alpha, int do_correct, int do_ghosts, int do_pg)
{
    k_project_run<real>(blockIdx, gridDim, G, Rg, Ru, Rv, Rw, K, u, v, w, pgu, pgv, pgw, phi, mc, mxy, mxz, myz, scal,
                        alpha, do_correct, do_ghosts, do_pg);
}
template <typename real>
struct k_project_b {
    static constexpr auto run = &k_project_run<real>;
    static constexpr int maxt = 128, minb = 0;
};

// The precision form's projection on cell pairs (k, k+32) with packed FP32x2
// arithmetic, as k_explicit2: the same fused correction, ghosts and pressure
// gradient as k_project, two cells per thread sharing their addresses (the
// second cell's are the first's plus 128 bytes) and their add / multiply /
// fma instructions.  A second cell past ke reads the slack past the arrays'
// ends and stores nothing.  Grid: x over k in tiles of 64 (blockDim.x 32).
template <int VAR, typename real>
__device__ __forceinline__ typename PairOf<real>::type pg_update2(const Consts& K, const Geo& G,
                                                                  const real* __restrict__ phi,
                                                                  const MuPtrs<real>& mu, long id,
                                                                  typename PairOf<real>::type fac,
                                                                  typename PairOf<real>::type pold)
{
    using T2 = typename PairOf<real>::type;
    const long sx = G.sx, sy = G.sy;
    const long so = VAR == VU ? sx : VAR == VV ? sy : 1;
    const T2 ih = S2((real)(VAR == VU ? K.ihx : VAR == VV ? K.ihy : K.ihz));
    auto gp = [&](long p) { return (ld2(phi, p) - ld2(phi, p - so)) * ih; };
    T2 a, b, c;
    const T2 g0 = gp(id);
    acoef2<VAR, 0, real>(K, G, mu, id, a, b, c);
    const T2 pxx = fma2(c, gp(id + sx), fma2(b, g0, a * gp(id - sx)));
    acoef2<VAR, 1, real>(K, G, mu, id, a, b, c);
    const T2 pyy = fma2(c, gp(id + sy), fma2(b, g0, a * gp(id - sy)));
    acoef2<VAR, 2, real>(K, G, mu, id, a, b, c);
    const T2 pzz = fma2(c, gp(id + 1), fma2(b, g0, a * gp(id - 1)));
    return pold + g0 - fac * (pyy + pxx + pzz);
}

template <typename real>
__device__ __forceinline__ void k_project2_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng Rg, Rng Ru, Rng Rv, Rng Rw,
        Consts K, real* __restrict__ u, real* __restrict__ v, real* __restrict__ w,
        real* __restrict__ pgu, real* __restrict__ pgv, real* __restrict__ pgw,
        const real* __restrict__ phi, MuPtrs<real> mu, const double* __restrict__ scal,
        double alpha, int do_correct, int do_ghosts, int do_pg)
{
    using T2 = typename PairOf<real>::type;
    const int k = Rg.ks + blockIdx.x * (2 * EP_DK) + threadIdx.x;
    const int j = Rg.js + blockIdx.y * blockDim.y + threadIdx.y;
    const int i = Rg.is + blockIdx.z;
    if (k > Rg.ke || j > Rg.je) return;
    const int kb = k + EP_DK;
    const bool live_b = kb <= Rg.ke;
    const long sx = G.sx, sy = G.sy;
    const long id = (long)i * sx + (long)j * sy + k;
    const double dt = scal[S_DT];
    // per cell: in the u / v / w ranges (the second cell's k is past every ks)
    const bool iu = (i >= Ru.is) & (i <= Ru.ie) & (j >= Ru.js);
    const bool iv = (i <= Rv.ie) & (j >= Rv.js), iw = (i <= Rw.ie) & (j >= Rw.js);
    const bool inu_a = iu & (k >= Ru.ks), inv_a = iv & (k >= Rv.ks), inw_a = iw & (k >= Rw.ks);
    const bool inu_b = iu & live_b, inv_b = iv & live_b, inw_b = iw & live_b;
    const bool ghost_i = (i <= Rg.ie);

    // ghost copies of one cell (k index kk, values after correction)
    auto ghosts = [&](long c, int kk, real uval, real vval, real wval) {
        if (kk == Rg.ks) { u[c - 1] = uval; v[c - 1] = vval; }
        if (kk == Rg.ke) { u[c + 1] = uval; v[c + 1] = vval; }
        if (j == Rg.js) { u[c - sy] = -uval; w[c - sy] = -wval; }
        if (j == Rg.je) { u[c + sy] = -uval; w[c + sy] = -wval; }
        if (i == Rg.is) { v[c - sx] = -vval; w[c - sx] = -wval; }
    };

    if (do_correct) {
        const T2 fac = S2((real)(dt * alpha / K.Re));
        T2 uval = ld2(u, id), vval = S2((real)0), wval = S2((real)0);
        if (ghost_i) {
            vval = ld2(v, id);
            wval = ld2(w, id);
        }
        const T2 p0 = ld2(phi, id);
        const T2 vn = vval - fac * ((p0 - ld2(phi, id - sy)) * S2((real)K.ihy));
        const T2 wn = wval - fac * ((p0 - ld2(phi, id - 1)) * S2((real)K.ihz));
        const T2 un = uval - fac * ((p0 - ld2(phi, id - sx)) * S2((real)K.ihx));
        if (inv_a) { v[id] = vn.v.x; vval.v.x = vn.v.x; }
        if (inv_b) { v[id + EP_DK] = vn.v.y; vval.v.y = vn.v.y; }
        if (inw_a) { w[id] = wn.v.x; wval.v.x = wn.v.x; }
        if (inw_b) { w[id + EP_DK] = wn.v.y; wval.v.y = wn.v.y; }
        if (inu_a) { u[id] = un.v.x; uval.v.x = un.v.x; }
        if (inu_b) { u[id + EP_DK] = un.v.y; uval.v.y = un.v.y; }
        if (i == Ru.ie + 1 && j >= Ru.js) {
            const real def = (real)scal[S_DEFICIT];
            if (k >= Ru.ks) u[id] = uval.v.x + def;
            if (live_b) u[id + EP_DK] = uval.v.y + def;
        }
        if (do_ghosts && ghost_i) {
            ghosts(id, k, uval.v.x, vval.v.x, wval.v.x);
            if (live_b) ghosts(id + EP_DK, kb, uval.v.y, vval.v.y, wval.v.y);
        }
    } else if (do_ghosts && ghost_i) {
        ghosts(id, k, u[id], v[id], w[id]);
        if (live_b) ghosts(id + EP_DK, kb, u[id + EP_DK], v[id + EP_DK], w[id + EP_DK]);
    }

    if (do_pg) {
        const T2 fac = S2((real)(0.5 * dt * alpha));
        if (inv_a | inv_b) {
            const T2 r = pg_update2<VV, real>(K, G, phi, mu, id, fac, ld2(pgv, id));
            if (inv_a) pgv[id] = r.v.x;
            if (inv_b) pgv[id + EP_DK] = r.v.y;
        }
        if (inu_a | inu_b) {
            const T2 r = pg_update2<VU, real>(K, G, phi, mu, id, fac, ld2(pgu, id));
            if (inu_a) pgu[id] = r.v.x;
            if (inu_b) pgu[id + EP_DK] = r.v.y;
        }
        if (inw_a | inw_b) {
            const T2 r = pg_update2<VW, real>(K, G, phi, mu, id, fac, ld2(pgw, id));
            if (inw_a) pgw[id] = r.v.x;
            if (inw_b) pgw[id + EP_DK] = r.v.y;
        }
    }
}
template <typename real>
__global__ void __launch_bounds__(128, sizeof(real) == 4 ? 16 : 8) k_project2(Geo G, Rng Rg, Rng Ru, Rng Rv, Rng Rw,
        Consts K, real* __restrict__ u, real* __restrict__ v, real* __restrict__ w,
        real* __restrict__ pgu, real* __restrict__ pgv, real* __restrict__ pgw,
        const real* __restrict__ phi, MuPtrs<real> mu, const double* __restrict__ scal,
        double alpha, int do_correct, int do_ghosts, int do_pg)
{
    k_project2_run<real>(blockIdx, gridDim, G, Rg, Ru, Rv, Rw, K, u, v, w, pgu, pgv, pgw, phi, mu, scal, alpha,
                         do_correct, do_ghosts, do_pg);
}
template <typename real>
struct k_project2_b {
    static constexpr auto run = &k_project2_run<real>;
    static constexpr int maxt = 128, minb = sizeof(real) == 4 ? 16 : 8, bminb = 8;
};

// The precision form's mode solve with a third of k_poisson_x's scratch
// traffic: the same FP64 Thomas recurrences per (ky, kz) mode, but the
// eliminated right-hand side is kept in FP32 (the mode data are FP32 on
// either side of the solve) and c' is not stored: it depends on the mode
// only, so the forward sweep records it every PX_CK rows and the backward
// sweep recomputes each block of PX_CK values from its checkpoint (the same
// arithmetic, so the same values).  One reciprocal per row and sweep instead
// of two divisions.  16.5 bytes per cell instead of 40.
constexpr int PX_CK = 16;

__device__ __forceinline__ void k_poisson_x2_run(const uint3 blockIdx, const dim3 gridDim,
    int nx, int ny, int nz, Consts K,
                                                    const double* __restrict__ lam_y,
                                                    const double* __restrict__ lam_z, float* __restrict__ hat,
                                                    float* __restrict__ rr, double* __restrict__ ck, int kz_major)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = ny * nz;
    if (t >= N) return;
    const int jy = kz_major ? t % ny : t / nz, kz = kz_major ? t / ny : t % nz;
    const long st = N;
    const double a = K.dx2i, c = K.dx2i;
    const double bmid = -2.0 * K.dx2i + lam_y[jy] + lam_z[kz];
    const bool gauge = (jy == 0) && (kz == 0);
    auto diag = [&](int m) {
        double lb = bmid;
        if (m == 0) lb += a;
        if (m == nx - 1 && !gauge) lb += c;
        return lb;
    };
    // forward: c'_m = c / (b_m - a c'_{m-1}), r'_m = (r_m - a r'_{m-1}) / (...)
    constexpr int PF = 8;
    double cprev = 0.0, rprev = 0.0;
    float hv[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) hv[u] = u < nx ? hat[t + (long)u * st] : 0.f;
    for (int m0 = 0; m0 < nx; m0 += PF) {
        float hn[PF];
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int m = m0 + PF + u;
            hn[u] = m < nx ? hat[t + (long)m * st] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int m = m0 + u;
            if (m < nx) {
                if (m % PX_CK == 0) ck[(long)(m / PX_CK) * st + t] = cprev;   // c'_{m-1}
                const double inv = 1.0 / (diag(m) - cprev * a);
                const double rm = ((double)hv[u] - rprev * a) * inv;
                cprev = c * inv;   // as the backward sweep recomputes it
                rprev = rm;
                rr[t + (long)m * st] = (float)rm;
            }
        }
#pragma unroll
        for (int u = 0; u < PF; ++u) hv[u] = hn[u];
    }
    // backward, one checkpoint block at a time from the end: x_{n-1} = r'_{n-1}
    double xnext = 0.0;
    for (int b0 = ((nx - 1) / PX_CK) * PX_CK; b0 >= 0; b0 -= PX_CK) {
        double cb[PX_CK];
        float rv[PX_CK];
        double cp = ck[(long)(b0 / PX_CK) * st + t];
#pragma unroll
        for (int u = 0; u < PX_CK; ++u) {
            const int m = b0 + u;
            rv[u] = m < nx ? rr[t + (long)m * st] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < PX_CK; ++u) {
            const int m = b0 + u;
            if (m < nx) cp = c * (1.0 / (diag(m) - cp * a));
            cb[u] = cp;
        }
#pragma unroll
        for (int u = PX_CK - 1; u >= 0; --u) {
            const int m = b0 + u;
            if (m < nx) {
                const double x = (m == nx - 1) ? (double)rv[u] : (double)rv[u] - cb[u] * xnext;
                hat[t + (long)m * st] = (float)x;
                xnext = x;
            }
        }
    }
}
__global__ void __launch_bounds__(128) k_poisson_x2(int nx, int ny, int nz, Consts K,
                                                    const double* __restrict__ lam_y,
                                                    const double* __restrict__ lam_z, float* __restrict__ hat,
                                                    float* __restrict__ rr, double* __restrict__ ck, int kz_major)
{
    k_poisson_x2_run(blockIdx, gridDim, nx, ny, nz, K, lam_y, lam_z, hat, rr, ck, kz_major);
}
struct k_poisson_x2_b {
    static constexpr auto run = &k_poisson_x2_run;
    static constexpr int maxt = 128, minb = 0;
};

// slope_parameter (pllcart3d.c:722-840) on one rank: bisection for the
// non-monotonic viscosity law's cm from c along the x line closest to
// y=0, z=0; also leaves the law's coefficients (L895-900) in the scalars.
// One thread.
static __global__ void k_slope_parameter(Geo G, Rng R, double Y1, double Z1, double dy, double dz,
                                  double M, double Mum, double Lambda, double PI,
                                  const double* __restrict__ cn, double* scal, int* status,
                                  double* work)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int n = R.ie - R.is + 1;
    double err = 10.0;
    int jj = R.js, kk = R.ks;
    for (int j = R.js; j <= R.je; ++j) {
        double yc = Y1 - R.js * dy + (dy / 2.0) + j * dy;
        if (fabs(yc - 0.0) < err) { err = fabs(yc - 0.0); jj = j; }
    }
    err = 10.0;
    for (int k = R.ks; k <= R.ke; ++k) {
        double zc = Z1 - R.ks * dz + (dz / 2.0) + k * dz;
        if (fabs(zc - 0.0) < err) { err = fabs(zc - 0.0); kk = k; }
    }
    double* croot = work;
    double* mucell = work + n;
    for (int i = R.is; i <= R.ie; ++i) croot[i - R.is] = cn[(long)i * G.sx + (long)jj * G.sy + kk];
    double alpha = exp(M), mum = Mum * alpha;
    double psi0 = asin(alpha / mum), psi1 = PI - asin(1 / mum);
    double etam = (PI / 2 - psi0) / (psi1 - psi0);
    double cL = 0.1, cH = 0.9, cm = 0.5 * (cL + cH), errd = 100, errl = 1e-5;
    int niter = 0, ok = 1;
    while (errd > 1e-5) {
        double a = ((1 - cm) - etam) / ((1 - cm) * (etam - 1));
        for (int i = 0; i < n; ++i) {
            double eta = ((1 + a) * croot[i]) / (1 + a * croot[i]);
            double psi = psi0 * (1 - eta) + psi1 * eta;
            mucell[i] = mum * sin(psi);
        }
        int idx1 = -1, idx2 = -1;
        for (int i = 0; i < n; ++i) {
            if (idx1 > 0) break;
            if (fabs(croot[i]) > errl) idx1 = i;
        }
        for (int i = n - 1; i >= 0; --i) {
            if (idx2 > 0) break;
            if (fabs(croot[i]) < 1 - errl) idx2 = i;
        }
        if (idx1 < 0 || idx2 < 1 || idx1 + 1 >= n) { ok = 0; break; }
        double mup1 = (mucell[idx1 + 1] - mucell[idx1]) / (croot[idx1 + 1] - croot[idx1]);
        double mup2 = (mucell[idx2] - mucell[idx2 - 1]) / (croot[idx2] - croot[idx2 - 1]);
        double lambda = (mup1 + mup2) / (alpha + 1);
        if (lambda > Lambda) cH = cm;
        else cL = cm;
        cm = 0.5 * (cL + cH);
        errd = fabs(lambda - Lambda);
        niter++;
        if (niter > 500) { ok = 0; break; }
    }
    if (!ok) atomicOr(status, (int)ST_NOCONV);
    scal[S_CM] = cm;
    scal[S_MUM] = mum;
    scal[S_PSI0] = psi0;
    scal[S_PSI1] = psi1;
    scal[S_NMVA] = ((1 - cm) - etam) / ((1 - cm) * (etam - 1));
}


// FP64 diagnostics of the state: per x-plane sums of c over the interior
// y-z plane (the yz mean of conc_average, pllcart3d.c:3692-3704) and the
// divergence of the new velocities, max |div| and sum div^2.  One block per
// x-plane; the plane sums are reduced in a fixed order (deterministic).
template <typename real>
__global__ void __launch_bounds__(256) k_plane_diag(Geo G, Rng R, Consts K, const real* __restrict__ c,
                                                    const real* __restrict__ u, const real* __restrict__ v,
                                                    const real* __restrict__ w, double* __restrict__ out)
{
    const int i = R.is + blockIdx.x;
    const int nj = R.je - R.js + 1, nk = R.ke - R.ks + 1;
    double sc = 0.0, dmax = 0.0, d2 = 0.0;
    for (int t = threadIdx.x; t < nj * nk; t += blockDim.x) {
        const int j = R.js + t / nk, k = R.ks + t % nk;
        const long id = (long)i * G.sx + (long)j * G.sy + k;
        sc += (double)c[id];
        const double dv = ((double)u[id + G.sx] - (double)u[id]) / K.hx +
                          ((double)v[id + G.sy] - (double)v[id]) / K.hy +
                          ((double)w[id + 1] - (double)w[id]) / K.hz;
        dmax = fmax(dmax, fabs(dv));
        d2 += dv * dv;
    }
    __shared__ double s0[256], s1[256], s2[256];
    s0[threadIdx.x] = sc;
    s1[threadIdx.x] = dmax;
    s2[threadIdx.x] = d2;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            s0[threadIdx.x] += s0[threadIdx.x + h];
            s1[threadIdx.x] = fmax(s1[threadIdx.x], s1[threadIdx.x + h]);
            s2[threadIdx.x] += s2[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[3 * blockIdx.x + 0] = s0[0];
        out[3 * blockIdx.x + 1] = s1[0];
        out[3 * blockIdx.x + 2] = s2[0];
    }
}

}  // namespace
}  // namespace pll
