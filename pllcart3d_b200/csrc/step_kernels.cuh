// Kernels of the pllcart3d RK3-CN step (pllcart3d.c:156-196), templated on
// the arithmetic type.  The FP64 instantiation is compiled without
// multiply-add contraction (--fmad=false) and keeps every division that the
// reference performs, except divisions by a grid spacing or by 4*ny*nz that
// is an exact power of two, which are exact multiplications by the exact
// reciprocal.  Operation order follows the reference expression by
// expression so that the FP64 path tracks it to rounding level.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

// 1: the exact FP64 form (the reference's divisions, in its order); 0: the
// FP64 form (WENO5 weights with one division).  Set by the form's
// translation unit; units that only share the types default to exact.
#ifndef PLL_FP64_EXACT
#define PLL_FP64_EXACT 1
#endif

namespace pll {
// internal linkage: each translation unit (and so each precision form with
// its own contraction flags) owns its instantiations
namespace {

enum { MU_CELL_ = 0, MU_XY_ = 1, MU_XZ_ = 2, MU_YZ_ = 3 };

// x / h as the reference divides; exact as x * (1/h) when h is a power of
// two.  The FP64 forms (within rounding of the reference, not its operation
// order) and the precision form always multiply by the rounded 1/h.
template <typename real>
__device__ __forceinline__ real over_h(real x, double h, double ih, int pow2)
{
#if PLL_FP64_EXACT
    return pow2 ? x * (real)ih : x / (real)h;
#else
    return x * (real)ih;
#endif
}

template <>
__device__ __forceinline__ float over_h<float>(float x, double, double ih, int)
{
    return x * (float)ih;
}

// x / (2 h), the ENO-2 second difference
template <typename real>
__device__ __forceinline__ real over_2h(real x, double h, double i2h, int pow2)
{
#if PLL_FP64_EXACT
    return pow2 ? x * (real)i2h : x / ((real)2.0 * (real)h);
#else
    return x * (real)i2h;
#endif
}

template <>
__device__ __forceinline__ float over_2h<float>(float x, double, double i2h, int)
{
    return x * (float)i2h;
}

// g a + r b, the RK combination of the explicit terms.  The exact form
// rounds both products and the sum as the reference does (it is compiled
// without contraction); the other forms fuse the first product and round
// the second on its own, so that the result does not depend on which of the
// two products a compiler would have fused.
__device__ __forceinline__ float mul_rn_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn_(double a, double b) { return __dmul_rn(a, b); }
template <typename real>
__device__ __forceinline__ real rk_comb(real g, real a, real r, real b)
{
#if PLL_FP64_EXACT
    if (sizeof(real) == 8) return g * a + r * b;
#endif
    return fma(g, a, mul_rn_(r, b));
}

// dt (g a + r b), the convective outflow increment of an x sweep: a rounded
// product outside the exact form, since it feeds both q_new = q_old + it and
// the last row's right-hand side (a product with two uses, which a compiler
// may fuse into either)
template <typename real>
__device__ __forceinline__ real rk_step(real dt, real g, real a, real r, real b)
{
#if PLL_FP64_EXACT
    if (sizeof(real) == 8) return dt * (g * a + r * b);
#endif
    return mul_rn_(dt, rk_comb<real>(g, a, r, b));
}

// advecting velocity of variable VAR for the pass along AXIS at point id
// (Hc_op L1563/1591/1621, Hu_op L1669/1696/1722, Hv_op L1780/1807/1834,
//  Hw_op L1892/1919/1946)
template <int VAR, int AXIS, typename real>
__device__ __forceinline__ real adv_vel(const real* __restrict__ self,
                                       const real* __restrict__ un,
                                       const real* __restrict__ vn,
                                       const real* __restrict__ wn, long id,
                                       long sx, long sy)
{
    const real h = (real)0.5, q = (real)0.25;
    if (VAR == VC) {
        if (AXIS == 0) return h * (un[id + sx] + un[id]);
        if (AXIS == 1) return h * (vn[id + sy] + vn[id]);
        return h * (wn[id + 1] + wn[id]);
    } else if (VAR == VU) {
        if (AXIS == 0) return self[id];
        if (AXIS == 1) return q * (vn[id - sx] + vn[id] + vn[id + sy] + vn[id - sx + sy]);
        return q * (wn[id - sx] + wn[id] + wn[id + 1] + wn[id - sx + 1]);
    } else if (VAR == VV) {
        if (AXIS == 0) return q * (un[id - sy] + un[id + sx - sy] + un[id] + un[id + sx]);
        if (AXIS == 1) return self[id];
        return q * (wn[id - sy] + wn[id - sy + 1] + wn[id] + wn[id + 1]);
    } else {
        if (AXIS == 0) return q * (un[id - 1] + un[id + sx - 1] + un[id] + un[id + sx]);
        if (AXIS == 1) return q * (vn[id - 1] + vn[id] + vn[id + sy - 1] + vn[id + sy]);
        return self[id];
    }
}

// WENO5 derivative from five divided differences (calculate_weno,
// pllcart3d.c:3455-3507)
template <typename real>
__device__ __forceinline__ real weno5(real v0, real v1, real v2, real v3, real v4)
{
    const real con1 = (real)(1.0 / 6.0), con2 = (real)(13.0 / 12.0), con3 = (real)(1.0 / 4.0);
    real maxd = (real)0, sq;
    sq = v0 * v0; maxd = (maxd > sq) ? maxd : sq;
    sq = v1 * v1; maxd = (maxd > sq) ? maxd : sq;
    sq = v2 * v2; maxd = (maxd > sq) ? maxd : sq;
    sq = v3 * v3; maxd = (maxd > sq) ? maxd : sq;
    sq = v4 * v4; maxd = (maxd > sq) ? maxd : sq;
    real c1 = con1 * ((real)2.0 * v0 - (real)7.0 * v1 + (real)11.0 * v2);
    real c2 = con1 * ((real)-1.0 * v1 + (real)5.0 * v2 + (real)2.0 * v3);
    real c3 = con1 * ((real)2.0 * v2 + (real)5.0 * v3 - (real)1.0 * v4);
    real t1 = v0 - (real)2.0 * v1 + (real)1.0 * v2;
    real t2 = v0 - (real)4.0 * v1 + (real)3.0 * v2;
    real s1 = (con2 * t1 * t1) + (con3 * t2 * t2);
    t1 = v1 - (real)2.0 * v2 + v3;
    t2 = v1 - v3;
    real s2 = (con2 * t1 * t1) + (con3 * t2 * t2);
    t1 = (real)1.0 * v2 - (real)2.0 * v3 + v4;
    t2 = (real)3.0 * v2 - (real)4.0 * v3 + v4;
    real s3 = (con2 * t1 * t1) + (con3 * t2 * t2);
    // FP64: the reference's 1e-99 floor.  FP32: 1e-99 underflows to 0 and
    // (s+eps)^2 could be 0; 1e-18 keeps (s+eps)^2 >= 1e-36, a normal float,
    // and below any smoothness indicator that matters
    real eps = (real)1.0e-6 * maxd + (sizeof(real) == 8 ? (real)1.0e-99 : (real)1.0e-18);
    real a1 = (real)0.1 / ((s1 + eps) * (s1 + eps));
    real a2 = (real)0.6 / ((s2 + eps) * (s2 + eps));
    real a3 = (real)0.3 / ((s3 + eps) * (s3 + eps));
    real at = a1 + a2 + a3;
    return (a1 / at) * c1 + (a2 / at) * c2 + (a3 / at) * c3;
}

#ifndef PLL_WENO_F32
#define PLL_WENO_F32 0
#endif

#if !PLL_FP64_EXACT && !PLL_WENO_F32
// The FP64 form's WENO5: the same nonlinear weights with one division.  The
// weights a_i = w_i / e_i^2 (e_i = s_i + eps) enter only through the ratio
// sum(a_i c_i) / sum(a_i), which is unchanged when every a_i is multiplied
// by (e_1 e_2 e_3)^2 f^6 for any f > 0; that leaves
// a_1 = w_1 (e_2 e_3 f^2)^2 and so on, with no division.  f = 2^-E, E the
// exponent of the largest e_i, is exact; since eps >= 1e-6 max(v^2) and every
// s_i <= 33 max(v^2), every e_i f lies in [1.5e-8, 2), so the products can
// neither underflow nor overflow.  The result agrees with the six-division
// sequence to rounding.
template <>
__device__ __forceinline__ double weno5<double>(double v0, double v1, double v2, double v3, double v4)
{
    const double con1 = 1.0 / 6.0, con2 = 13.0 / 12.0, con3 = 0.25;
    const double maxd = fmax(fmax(fmax(v0 * v0, v1 * v1), fmax(v2 * v2, v3 * v3)), v4 * v4);
    const double c1 = con1 * (2.0 * v0 - 7.0 * v1 + 11.0 * v2);
    const double c2 = con1 * (-v1 + 5.0 * v2 + 2.0 * v3);
    const double c3 = con1 * (2.0 * v2 + 5.0 * v3 - v4);
    double t1 = v0 - 2.0 * v1 + v2, t2 = v0 - 4.0 * v1 + 3.0 * v2;
    const double s1 = con2 * t1 * t1 + con3 * t2 * t2;
    t1 = v1 - 2.0 * v2 + v3;
    t2 = v1 - v3;
    const double s2 = con2 * t1 * t1 + con3 * t2 * t2;
    t1 = v2 - 2.0 * v3 + v4;
    t2 = 3.0 * v2 - 4.0 * v3 + v4;
    const double s3 = con2 * t1 * t1 + con3 * t2 * t2;
    const double eps = 1.0e-6 * maxd + 1.0e-99;
    double e1 = s1 + eps, e2 = s2 + eps, e3 = s3 + eps;
    const long long be = __double_as_longlong(fmax(fmax(e1, e2), e3)) >> 52;   // biased exponent, e > 0
    const double f = __longlong_as_double((2046LL - be) << 52);                 // 2^-(be - 1023)
    e1 *= f;
    e2 *= f;
    e3 *= f;
    const double p23 = e2 * e3, p13 = e1 * e3, p12 = e1 * e2;
    const double a1 = 0.1 * (p23 * p23), a2 = 0.6 * (p13 * p13), a3 = 0.3 * (p12 * p12);
    return (a1 * c1 + a2 * c2 + a3 * c3) / (a1 + a2 + a3);
}
#endif

// The precision form's WENO5: the same weights with four approximate
// divisions (__fdividef, <= 2 ulp) in place of six IEEE ones.  With the FP32
// floor eps >= 1e-18 every (s+eps)^2 lies in [1e-36, 2^126), where
// __fdividef is accurate, and so does the weight sum.
template <>
__device__ __forceinline__ float weno5<float>(float v0, float v1, float v2, float v3, float v4)
{
    const float con1 = (float)(1.0 / 6.0), con2 = (float)(13.0 / 12.0), con3 = 0.25f;
    const float maxd = fmaxf(fmaxf(fmaxf(v0 * v0, v1 * v1), fmaxf(v2 * v2, v3 * v3)), v4 * v4);
    const float c1 = con1 * (2.0f * v0 - 7.0f * v1 + 11.0f * v2);
    const float c2 = con1 * (-v1 + 5.0f * v2 + 2.0f * v3);
    const float c3 = con1 * (2.0f * v2 + 5.0f * v3 - v4);
    float t1 = v0 - 2.0f * v1 + v2, t2 = v0 - 4.0f * v1 + 3.0f * v2;
    const float s1 = con2 * t1 * t1 + con3 * t2 * t2;
    t1 = v1 - 2.0f * v2 + v3;
    t2 = v1 - v3;
    const float s2 = con2 * t1 * t1 + con3 * t2 * t2;
    t1 = v2 - 2.0f * v3 + v4;
    t2 = 3.0f * v2 - 4.0f * v3 + v4;
    const float s3 = con2 * t1 * t1 + con3 * t2 * t2;
    const float eps = 1.0e-6f * maxd + 1.0e-18f;
    const float a1 = __fdividef(0.1f, (s1 + eps) * (s1 + eps));
    const float a2 = __fdividef(0.6f, (s2 + eps) * (s2 + eps));
    const float a3 = __fdividef(0.3f, (s3 + eps) * (s3 + eps));
    return __fdividef(a1 * c1 + a2 * c2 + a3 * c3, a1 + a2 + a3);
}

#if !PLL_FP64_EXACT && PLL_WENO_F32
// The FP64-state form's WENO5: the five FP64 divided differences rounded to
// FP32 once, the smoothness indicators, weights and weighted sum in FP32
// (weno5<float>), the result widened back.  Relative error of the derivative
// ~1e-7; every other operation of the step stays FP64.
template <>
__device__ __forceinline__ double weno5<double>(double v0, double v1, double v2, double v3, double v4)
{
    return (double)weno5<float>((float)v0, (float)v1, (float)v2, (float)v3, (float)v4);
}
#endif

// D2 value an earlier directional pass of the same H*_op call left in its
// scratch line at index m (pllcart3d.c:1545-1546: D1/D2 are allocated once
// per call, zeroed, and reused by the x, y and z passes; each pass writes
// D2 only on the variable's own range, so the ENO-2 closure reads one point
// outside the range pick up the previous pass's last line).  The x pass
// leaves (j=je, k=ke), the y pass (i=ie, k=ke).
template <typename real>
__device__ real stale_d2(const real* __restrict__ q, const Geo& G, const Rng& R,
                         const Consts& K, int pass, int m)
{
    for (int p = pass - 1; p >= 0; --p) {
        int s = p == 0 ? R.is : R.js, e = p == 0 ? R.ie : R.je;
        if (m >= s && m <= e) {
            long base, st;
            double h, ih, i2h;
            if (p == 0) {
                base = (long)R.je * G.sy + R.ke; st = G.sx; h = K.hx; ih = K.ihx; i2h = K.i2hx;
            } else {
                base = (long)R.ie * G.sx + R.ke; st = G.sy; h = K.hy; ih = K.ihy; i2h = K.i2hy;
            }
            real d1m = over_h<real>(q[base + (long)(m + 1) * st] - q[base + (long)m * st], h, ih, K.pow2);
            real d1p = over_h<real>(q[base + (long)m * st] - q[base + (long)(m - 1) * st], h, ih, K.pow2);
            return over_2h<real>(d1m - d1p, h, i2h, K.pow2);
        }
    }
    return (real)0;
}

// c' = c / b', r' = r / b' of one Thomas step: the exact form divides
// twice as the reference does; the FP64 forms divide once and multiply by
// the reciprocal; the precision form multiplies by one approximate
// reciprocal (b' >= 1 for these diagonally dominant systems, so __fdividef
// is accurate to 2 ulp).
template <typename real>
__device__ __forceinline__ void thomas_div(real lc, real num, real bb, real& cm, real& rm)
{
#if !PLL_FP64_EXACT
    const real ib = (real)1 / bb;
    cm = lc * ib;
    rm = num * ib;
#else
    cm = lc / bb;
    rm = num / bb;
#endif
}

template <>
__device__ __forceinline__ void thomas_div<float>(float lc, float num, float bb, float& cm, float& rm)
{
    const float ib = __fdividef(1.0f, bb);
    cm = lc * ib;
    rm = num * ib;
}

// upwind derivative of q along AXIS at point id (line position m); the
// ENO-2 closure on the first and last two points of the range, WENO5
// elsewhere (e.g. Hc_op pllcart3d.c:1553-1576)
template <int AXIS, typename real>
__device__ __forceinline__ real upwind_deriv(const real* __restrict__ q, const Geo& G,
                                             const Rng& R, const Consts& K, long id,
                                             int m, real vv)
{
    const int s = AXIS == 0 ? R.is : AXIS == 1 ? R.js : R.ks;
    const int e = AXIS == 0 ? R.ie : AXIS == 1 ? R.je : R.ke;
    const long st = AXIS == 0 ? G.sx : AXIS == 1 ? G.sy : 1;
    const double h = AXIS == 0 ? K.hx : AXIS == 1 ? K.hy : K.hz;
    const double ih = AXIS == 0 ? K.ihx : AXIS == 1 ? K.ihy : K.ihz;
    const double i2h = AXIS == 0 ? K.i2hx : AXIS == 1 ? K.i2hy : K.i2hz;
    const int sign = (vv >= (real)0) ? 1 : -1;
    if ((m <= s + 1) | (m >= e - 1)) {
        const int kk = (sign == 1) ? m - 1 : m;
        const long b = id + (long)(kk - m) * st;
        real d1k = over_h<real>(q[b + st] - q[b], h, ih, K.pow2);
        real d2a, d2b;
        if (kk >= s) {
            real d1m = over_h<real>(q[b] - q[b - st], h, ih, K.pow2);
            d2a = over_2h<real>(d1k - d1m, h, i2h, K.pow2);
        } else {
            d2a = stale_d2<real>(q, G, R, K, AXIS, kk);
        }
        if (kk + 1 <= e) {
            real d1p = over_h<real>(q[b + 2 * st] - q[b + st], h, ih, K.pow2);
            d2b = over_2h<real>(d1p - d1k, h, i2h, K.pow2);
        } else {
            d2b = stale_d2<real>(q, G, R, K, AXIS, kk + 1);
        }
        real d2v = (fabs(d2a) <= fabs(d2b)) ? d2a : d2b;
        return d1k + d2v * (real)h * (real)sign;
    }
    // WENO: D1[kk + sign*t], t = 0..4, kk = m-3 (sign>0) or m+2 (sign<0).
    // Both windows lie in D1[m-3 .. m+2]: form those six differences from
    // q[m-3 .. m+3] at fixed offsets and pick the window by the sign.
    real d[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        const long p = id + (long)(t - 3) * st;
        d[t] = over_h<real>(q[p + st] - q[p], h, ih, K.pow2);
    }
    const bool up = sign == 1;
    return weno5<real>(up ? d[0] : d[5], up ? d[1] : d[4], up ? d[2] : d[3], up ? d[3] : d[2], up ? d[4] : d[1]);
}

// implicit-operator coefficients (A_conc/A_umom/A_vmom/A_wmom,
// pllcart3d.c:1411-1536) from the viscosity arrays
template <int VAR, int AXIS, typename real>
__device__ __forceinline__ void acoef(const Consts& K, const Geo& G,
                                      const real* __restrict__ mc,
                                      const real* __restrict__ mxy,
                                      const real* __restrict__ mxz,
                                      const real* __restrict__ myz, long id,
                                      real& a, real& b, real& c)
{
    const long sx = G.sx, sy = G.sy;
    if (VAR == VC) {
        const real d = (real)(AXIS == 0 ? K.cdx : AXIS == 1 ? K.cdy : K.cdz);
        a = d;
        c = d;
    } else if (VAR == VU) {
        if (AXIS == 0) {
            a = over_h<real>((real)K.d2x * mc[id - sx], K.hx, K.ihx, K.pow2);
            c = over_h<real>((real)K.d2x * mc[id], K.hx, K.ihx, K.pow2);
        } else if (AXIS == 1) {
            a = over_h<real>((real)K.d1y * mxy[id], K.hy, K.ihy, K.pow2);
            c = over_h<real>((real)K.d1y * mxy[id + sy], K.hy, K.ihy, K.pow2);
        } else {
            a = over_h<real>((real)K.d1z * mxz[id], K.hz, K.ihz, K.pow2);
            c = over_h<real>((real)K.d1z * mxz[id + 1], K.hz, K.ihz, K.pow2);
        }
    } else if (VAR == VV) {
        if (AXIS == 0) {
            a = over_h<real>((real)K.d1x * mxy[id], K.hx, K.ihx, K.pow2);
            c = over_h<real>((real)K.d1x * mxy[id + sx], K.hx, K.ihx, K.pow2);
        } else if (AXIS == 1) {
            a = over_h<real>((real)K.d2y * mc[id - sy], K.hy, K.ihy, K.pow2);
            c = over_h<real>((real)K.d2y * mc[id], K.hy, K.ihy, K.pow2);
        } else {
            a = over_h<real>((real)K.d1z * myz[id], K.hz, K.ihz, K.pow2);
            c = over_h<real>((real)K.d1z * myz[id + 1], K.hz, K.ihz, K.pow2);
        }
    } else {
        if (AXIS == 0) {
            a = over_h<real>((real)K.d1x * mxz[id], K.hx, K.ihx, K.pow2);
            c = over_h<real>((real)K.d1x * mxz[id + sx], K.hx, K.ihx, K.pow2);
        } else if (AXIS == 1) {
            a = over_h<real>((real)K.d1y * myz[id], K.hy, K.ihy, K.pow2);
            c = over_h<real>((real)K.d1y * myz[id + sy], K.hy, K.ihy, K.pow2);
        } else {
            a = over_h<real>((real)K.d2z * mc[id - 1], K.hz, K.ihz, K.pow2);
            c = over_h<real>((real)K.d2z * mc[id], K.hz, K.ihz, K.pow2);
        }
    }
    b = -(a + c);
}

template <typename real>
struct ExplicitArgs {
    const real* q;      // q_old of the variable
    const real* un;     // advecting / cross-term velocities
    const real* vn;
    const real* wn;
    MuPtrs<real> mu;    // mu_old
    const real* cn;     // c_new (body force of u and v)
    const real* pg;     // accumulated pressure gradient of the variable
    const real* Hm;     // explicit term of the previous substep
    real* H;            // explicit term of this substep (out)
    real* S;            // right-hand side of the ADI solve (out)
    const double* scal; // device scalars (dt)
    double g, r, alpha; // RK3 gamma, rho and gamma+rho
};

// ---------------------------------------------------------------------------
// explicit operator + right-hand side of one variable
// Hc_op/Hu_op/Hv_op/Hw_op (pllcart3d.c:1539-1980) fused with the source
// assembly of concentration/xmom/ymom/zmom (L573-590, L970-989, L1127-1146,
// L1280-1298)
// ---------------------------------------------------------------------------
template <int VAR, typename real>
__device__ __forceinline__ void k_explicit_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K,
                                                  ExplicitArgs<real> A)
{
    const int k = R.ks + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = R.js + blockIdx.y * blockDim.y + threadIdx.y;
    const int i = R.is + blockIdx.z;
    if (k > R.ke || j > R.je) return;
    const long sx = G.sx, sy = G.sy;
    const long id = (long)i * sx + (long)j * sy + k;
    const real* __restrict__ q = A.q;

    real vx = adv_vel<VAR, 0, real>(q, A.un, A.vn, A.wn, id, sx, sy);
    real cx = vx * upwind_deriv<0, real>(q, G, R, K, id, i, vx);
    real vy = adv_vel<VAR, 1, real>(q, A.un, A.vn, A.wn, id, sx, sy);
    real cy = vy * upwind_deriv<1, real>(q, G, R, K, id, j, vy);
    real vz = adv_vel<VAR, 2, real>(q, A.un, A.vn, A.wn, id, sx, sy);
    real cz = vz * upwind_deriv<2, real>(q, G, R, K, id, k, vz);
    real ct = cz + cx + cy;
    real H;
    if (VAR == VC) {
        H = -(ct);
    } else {
        const real* __restrict__ un = A.un;
        const real* __restrict__ vn = A.vn;
        const real* __restrict__ wn = A.wn;
        real s1, s2, s3, s4;
        if (VAR == VU) {
            s1 = (real)K.xuv * A.mu.xy[id + sy] * (vn[id + sy] - vn[id - sx + sy]);
            s2 = (real)K.xuv * A.mu.xy[id] * (vn[id] - vn[id - sx]);
            s3 = (real)K.xuw * A.mu.xz[id + 1] * (wn[id + 1] - wn[id - sx + 1]);
            s4 = (real)K.xuw * A.mu.xz[id] * (wn[id] - wn[id - sx]);
        } else if (VAR == VV) {
            s1 = (real)K.xvu * A.mu.xy[id + sx] * (un[id + sx] - un[id + sx - sy]);
            s2 = (real)K.xvu * A.mu.xy[id] * (un[id] - un[id - sy]);
            s3 = (real)K.xvw * A.mu.yz[id + 1] * (wn[id + 1] - wn[id - sy + 1]);
            s4 = (real)K.xvw * A.mu.yz[id] * (wn[id] - wn[id - sy]);
        } else {
            s1 = (real)K.xwu * A.mu.xz[id + sx] * (un[id + sx] - un[id + sx - 1]);
            s2 = (real)K.xwu * A.mu.xz[id] * (un[id] - un[id - 1]);
            s3 = (real)K.xwv * A.mu.yz[id + sy] * (vn[id + sy] - vn[id + sy - 1]);
            s4 = (real)K.xwv * A.mu.yz[id] * (vn[id] - vn[id - 1]);
        }
        H = -ct + s1 - s2 + s3 - s4;
    }
    A.H[id] = H;

    // right-hand side dt*(gamma H + rho H_old + alpha A q_old + alpha body)
    const real dt = (real)A.scal[S_DT];
    const real alpha = (real)A.alpha;
    real conv = rk_comb<real>((real)A.g, H, (real)A.r, A.Hm[id]);
    real a, b, c;
    acoef<VAR, 0, real>(K, G, A.mu.cell, A.mu.xy, A.mu.xz, A.mu.yz, id, a, b, c);
    real ax = a * q[id - sx] + b * q[id] + c * q[id + sx];
    acoef<VAR, 1, real>(K, G, A.mu.cell, A.mu.xy, A.mu.xz, A.mu.yz, id, a, b, c);
    real ay = a * q[id - sy] + b * q[id] + c * q[id + sy];
    acoef<VAR, 2, real>(K, G, A.mu.cell, A.mu.xy, A.mu.xz, A.mu.yz, id, a, b, c);
    real az = a * q[id - 1] + b * q[id] + c * q[id + 1];
    real diff = alpha * (ax + ay + az);
    real S;
    if (VAR == VC) {
        S = dt * (conv + diff);
    } else {
        real bf;
        if (VAR == VU) {
            real cval = (real)0.5 * (A.cn[id] + A.cn[id - sx]);
            bf = alpha * ((real)K.FxRe * cval - over_h<real>(A.pg[id], K.Re, 1.0 / K.Re, 0));
        } else if (VAR == VV) {
            real cval = (real)0.5 * (A.cn[id] + A.cn[id - sy]);
            bf = alpha * ((real)K.FyRe * cval - over_h<real>(A.pg[id], K.Re, 1.0 / K.Re, 0));
        } else {
            bf = alpha * (-over_h<real>(A.pg[id], K.Re, 1.0 / K.Re, 0));
        }
        S = dt * (conv + diff + bf);
    }
    A.S[id] = S;
}
template <int VAR, typename real>
__global__ void __launch_bounds__(128) k_explicit(Geo G, Rng R, Consts K,
                                                  ExplicitArgs<real> A)
{
    k_explicit_run<VAR, real>(blockIdx, gridDim, G, R, K, A);
}
template <int VAR, typename real>
struct k_explicit_b {
    static constexpr auto run = &k_explicit_run<VAR, real>;
    static constexpr int maxt = 128, minb = 0;
};

// ---------------------------------------------------------------------------
// The precision form's explicit operator on cell pairs with packed FP32x2
// arithmetic.  k_explicit in FP32 is issue-bound (~620 instructions per
// cell, 40 % of them FP32 add / multiply / fma), so each thread takes two
// cells, (i, j, k) and (i, j, k + 32), and runs the shared arithmetic once on
// both through sm_100's paired instructions (__fadd2_rn / __fmul2_rn /
// __ffma2_rn, one instruction for two FP32 operations); the second cell's
// loads are the first cell's addresses plus 128 bytes, so its address
// arithmetic is free too.  Every formula, constant and closure is
// k_explicit's; the two differ only in where a multiply and an add are fused
// (FP32 rounding level).  Points past the line's end: the second cell of the
// last tile may lie past ke; it is computed from reads into the row beyond
// (every device array carries zeroed slack past its end for this) and never
// stored.
// ---------------------------------------------------------------------------
struct f2 {
    float2 v;
};
__device__ __forceinline__ f2 F2(float a, float b) { return f2{make_float2(a, b)}; }
__device__ __forceinline__ f2 S2(float a) { return f2{make_float2(a, a)}; }
__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return f2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ f2 operator*(f2 a, f2 b) { return f2{__fmul2_rn(a.v, b.v)}; }
// a - b, and a + b * c, with one rounding each
__device__ __forceinline__ f2 operator-(f2 a, f2 b) { return f2{__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ f2 fma2(f2 b, f2 c, f2 a) { return f2{__ffma2_rn(b.v, c.v, a.v)}; }
__device__ __forceinline__ f2 neg2(f2 a) { return a * S2(-1.f); }

constexpr int EP_DK = 32;   // k distance of a thread's two cells

__device__ __forceinline__ f2 ld2(const float* __restrict__ p, long id) { return F2(p[id], p[id + EP_DK]); }

// the same cell pairs in FP64 (used by the FP64 forms): each operation is
// two scalar FP64 operations, the pair sharing its addressing
struct d2 {
    double2 v;
};
__device__ __forceinline__ d2 D2(double a, double b) { return d2{make_double2(a, b)}; }
__device__ __forceinline__ d2 S2(double a) { return D2(a, a); }
__device__ __forceinline__ d2 operator+(d2 a, d2 b) { return D2(a.v.x + b.v.x, a.v.y + b.v.y); }
__device__ __forceinline__ d2 operator*(d2 a, d2 b) { return D2(a.v.x * b.v.x, a.v.y * b.v.y); }
__device__ __forceinline__ d2 operator-(d2 a, d2 b) { return D2(a.v.x - b.v.x, a.v.y - b.v.y); }
__device__ __forceinline__ d2 fma2(d2 b, d2 c, d2 a) { return D2(fma(b.v.x, c.v.x, a.v.x), fma(b.v.y, c.v.y, a.v.y)); }
__device__ __forceinline__ d2 neg2(d2 a) { return D2(-a.v.x, -a.v.y); }
__device__ __forceinline__ d2 ld2(const double* __restrict__ p, long id) { return D2(p[id], p[id + EP_DK]); }
__device__ __forceinline__ f2 mk2(float a, float b) { return F2(a, b); }
__device__ __forceinline__ d2 mk2(double a, double b) { return D2(a, b); }

// the pair type of an arithmetic type
template <typename real>
struct PairOf {
    using type = f2;
};
template <>
struct PairOf<double> {
    using type = d2;
};

// packed weno5<float>: the same weights with the approximate divisions per
// component
__device__ __forceinline__ f2 weno5_2(f2 v0, f2 v1, f2 v2, f2 v3, f2 v4)
{
    const f2 con1 = S2((float)(1.0 / 6.0)), con2 = S2((float)(13.0 / 12.0)), con3 = S2(0.25f);
    const f2 q0 = v0 * v0, q1 = v1 * v1, q2 = v2 * v2, q3 = v3 * v3, q4 = v4 * v4;
    const f2 maxd = F2(fmaxf(fmaxf(fmaxf(q0.v.x, q1.v.x), fmaxf(q2.v.x, q3.v.x)), q4.v.x),
                       fmaxf(fmaxf(fmaxf(q0.v.y, q1.v.y), fmaxf(q2.v.y, q3.v.y)), q4.v.y));
    const f2 c1 = con1 * fma2(S2(2.0f), v0, fma2(S2(-7.0f), v1, S2(11.0f) * v2));
    const f2 c2 = con1 * fma2(S2(2.0f), v3, fma2(S2(5.0f), v2, neg2(v1)));
    const f2 c3 = con1 * fma2(S2(2.0f), v2, fma2(S2(5.0f), v3, neg2(v4)));
    f2 t1 = fma2(S2(-2.0f), v1, v0) + v2, t2 = fma2(S2(3.0f), v2, fma2(S2(-4.0f), v1, v0));
    const f2 s1 = fma2(con2 * t1, t1, con3 * t2 * t2);
    t1 = fma2(S2(-2.0f), v2, v1) + v3;
    t2 = v1 - v3;
    const f2 s2 = fma2(con2 * t1, t1, con3 * t2 * t2);
    t1 = fma2(S2(-2.0f), v3, v2) + v4;
    t2 = fma2(S2(-4.0f), v3, S2(3.0f) * v2) + v4;
    const f2 s3 = fma2(con2 * t1, t1, con3 * t2 * t2);
    const f2 eps = fma2(S2(1.0e-6f), maxd, S2(1.0e-18f));
    const f2 e1 = s1 + eps, e2 = s2 + eps, e3 = s3 + eps;
    const f2 d1 = e1 * e1, d2 = e2 * e2, d3 = e3 * e3;
    const f2 a1 = S2(0.1f) * F2(__fdividef(1.0f, d1.v.x), __fdividef(1.0f, d1.v.y));
    const f2 a2 = S2(0.6f) * F2(__fdividef(1.0f, d2.v.x), __fdividef(1.0f, d2.v.y));
    const f2 a3 = S2(0.3f) * F2(__fdividef(1.0f, d3.v.x), __fdividef(1.0f, d3.v.y));
    const f2 num = fma2(a3, c3, fma2(a2, c2, a1 * c1));
    const f2 den = a1 + a2 + a3;
    return num * F2(__fdividef(1.0f, den.v.x), __fdividef(1.0f, den.v.y));
}

template <int VAR, int AXIS>
__device__ __forceinline__ f2 adv_vel2(const float* __restrict__ self, const float* __restrict__ un,
                                       const float* __restrict__ vn, const float* __restrict__ wn, long id, long sx,
                                       long sy)
{
    const f2 h = S2(0.5f), q = S2(0.25f);
    if (VAR == VC) {
        if (AXIS == 0) return h * (ld2(un, id + sx) + ld2(un, id));
        if (AXIS == 1) return h * (ld2(vn, id + sy) + ld2(vn, id));
        return h * (ld2(wn, id + 1) + ld2(wn, id));
    } else if (VAR == VU) {
        if (AXIS == 0) return ld2(self, id);
        if (AXIS == 1) return q * (ld2(vn, id - sx) + ld2(vn, id) + ld2(vn, id + sy) + ld2(vn, id - sx + sy));
        return q * (ld2(wn, id - sx) + ld2(wn, id) + ld2(wn, id + 1) + ld2(wn, id - sx + 1));
    } else if (VAR == VV) {
        if (AXIS == 0) return q * (ld2(un, id - sy) + ld2(un, id + sx - sy) + ld2(un, id) + ld2(un, id + sx));
        if (AXIS == 1) return ld2(self, id);
        return q * (ld2(wn, id - sy) + ld2(wn, id - sy + 1) + ld2(wn, id) + ld2(wn, id + 1));
    } else {
        if (AXIS == 0) return q * (ld2(un, id - 1) + ld2(un, id + sx - 1) + ld2(un, id) + ld2(un, id + sx));
        if (AXIS == 1) return q * (ld2(vn, id - 1) + ld2(vn, id) + ld2(vn, id + sy - 1) + ld2(vn, id + sy));
        return ld2(self, id);
    }
}

// upwind derivative of both cells along AXIS; m is the first cell's line
// position (the second's is m + EP_DK along z, m along x and y).  Pairs with
// a cell in the ENO-2 band take upwind_deriv per cell.
template <int AXIS>
__device__ __forceinline__ f2 upwind_deriv2(const float* __restrict__ q, const Geo& G, const Rng& R,
                                            const Consts& K, long id, int m, f2 vv)
{
    const int s = AXIS == 0 ? R.is : AXIS == 1 ? R.js : R.ks;
    const int e = AXIS == 0 ? R.ie : AXIS == 1 ? R.je : R.ke;
    const int mb = AXIS == 2 ? m + EP_DK : m;
    const bool eno = (m <= s + 1) | (m >= e - 1) | (mb <= s + 1) | (mb >= e - 1);
    if (eno)
        return F2(upwind_deriv<AXIS, float>(q, G, R, K, id, m, vv.v.x),
                  upwind_deriv<AXIS, float>(q, G, R, K, id + EP_DK, mb, vv.v.y));
    const long st = AXIS == 0 ? G.sx : AXIS == 1 ? G.sy : 1;
    const f2 ih = S2((float)(AXIS == 0 ? K.ihx : AXIS == 1 ? K.ihy : K.ihz));
    f2 d[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        const long p = id + (long)(t - 3) * st;
        d[t] = (ld2(q, p + st) - ld2(q, p)) * ih;
    }
    const bool ua = vv.v.x >= 0.f, ub = vv.v.y >= 0.f;
    auto pick = [&](int up, int dn) { return F2(ua ? d[up].v.x : d[dn].v.x, ub ? d[up].v.y : d[dn].v.y); };
    return weno5_2(pick(0, 5), pick(1, 4), pick(2, 3), pick(3, 2), pick(4, 1));
}

template <int VAR, int AXIS, typename real>
__device__ __forceinline__ void acoef2(const Consts& K, const Geo& G, const MuPtrs<real>& mu, long id,
                                       typename PairOf<real>::type& a, typename PairOf<real>::type& b,
                                       typename PairOf<real>::type& c)
{
    using T2 = typename PairOf<real>::type;
    const long sx = G.sx, sy = G.sy;
    const T2 ihx = S2((real)K.ihx), ihy = S2((real)K.ihy), ihz = S2((real)K.ihz);
    if (VAR == VC) {
        a = c = S2((real)(AXIS == 0 ? K.cdx : AXIS == 1 ? K.cdy : K.cdz));
    } else if (VAR == VU) {
        if (AXIS == 0) {
            a = S2((real)K.d2x) * ld2(mu.cell, id - sx) * ihx;
            c = S2((real)K.d2x) * ld2(mu.cell, id) * ihx;
        } else if (AXIS == 1) {
            a = S2((real)K.d1y) * ld2(mu.xy, id) * ihy;
            c = S2((real)K.d1y) * ld2(mu.xy, id + sy) * ihy;
        } else {
            a = S2((real)K.d1z) * ld2(mu.xz, id) * ihz;
            c = S2((real)K.d1z) * ld2(mu.xz, id + 1) * ihz;
        }
    } else if (VAR == VV) {
        if (AXIS == 0) {
            a = S2((real)K.d1x) * ld2(mu.xy, id) * ihx;
            c = S2((real)K.d1x) * ld2(mu.xy, id + sx) * ihx;
        } else if (AXIS == 1) {
            a = S2((real)K.d2y) * ld2(mu.cell, id - sy) * ihy;
            c = S2((real)K.d2y) * ld2(mu.cell, id) * ihy;
        } else {
            a = S2((real)K.d1z) * ld2(mu.yz, id) * ihz;
            c = S2((real)K.d1z) * ld2(mu.yz, id + 1) * ihz;
        }
    } else {
        if (AXIS == 0) {
            a = S2((real)K.d1x) * ld2(mu.xz, id) * ihx;
            c = S2((real)K.d1x) * ld2(mu.xz, id + sx) * ihx;
        } else if (AXIS == 1) {
            a = S2((real)K.d1y) * ld2(mu.yz, id) * ihy;
            c = S2((real)K.d1y) * ld2(mu.yz, id + sy) * ihy;
        } else {
            a = S2((real)K.d2z) * ld2(mu.cell, id - 1) * ihz;
            c = S2((real)K.d2z) * ld2(mu.cell, id) * ihz;
        }
    }
    b = neg2(a + c);
}

// grid: x over k in tiles of 2 * EP_DK (blockDim.x == EP_DK), y over j, z over i
template <int VAR>
__device__ __forceinline__ void k_explicit2_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, ExplicitArgs<float> A)
{
    const int k = R.ks + blockIdx.x * (2 * EP_DK) + threadIdx.x;
    const int j = R.js + blockIdx.y * blockDim.y + threadIdx.y;
    const int i = R.is + blockIdx.z;
    if (k > R.ke || j > R.je) return;
    const bool live_b = k + EP_DK <= R.ke;
    const long sx = G.sx, sy = G.sy;
    const long id = (long)i * sx + (long)j * sy + k;
    const float* __restrict__ q = A.q;

    const f2 vx = adv_vel2<VAR, 0>(q, A.un, A.vn, A.wn, id, sx, sy);
    const f2 cx = vx * upwind_deriv2<0>(q, G, R, K, id, i, vx);
    const f2 vy = adv_vel2<VAR, 1>(q, A.un, A.vn, A.wn, id, sx, sy);
    const f2 cy = vy * upwind_deriv2<1>(q, G, R, K, id, j, vy);
    const f2 vz = adv_vel2<VAR, 2>(q, A.un, A.vn, A.wn, id, sx, sy);
    const f2 cz = vz * upwind_deriv2<2>(q, G, R, K, id, k, vz);
    const f2 ct = cz + cx + cy;
    f2 H;
    if (VAR == VC) {
        H = neg2(ct);
    } else {
        const float* __restrict__ un = A.un;
        const float* __restrict__ vn = A.vn;
        const float* __restrict__ wn = A.wn;
        f2 s1, s2, s3, s4;
        if (VAR == VU) {
            s1 = S2((float)K.xuv) * ld2(A.mu.xy, id + sy) * (ld2(vn, id + sy) - ld2(vn, id - sx + sy));
            s2 = S2((float)K.xuv) * ld2(A.mu.xy, id) * (ld2(vn, id) - ld2(vn, id - sx));
            s3 = S2((float)K.xuw) * ld2(A.mu.xz, id + 1) * (ld2(wn, id + 1) - ld2(wn, id - sx + 1));
            s4 = S2((float)K.xuw) * ld2(A.mu.xz, id) * (ld2(wn, id) - ld2(wn, id - sx));
        } else if (VAR == VV) {
            s1 = S2((float)K.xvu) * ld2(A.mu.xy, id + sx) * (ld2(un, id + sx) - ld2(un, id + sx - sy));
            s2 = S2((float)K.xvu) * ld2(A.mu.xy, id) * (ld2(un, id) - ld2(un, id - sy));
            s3 = S2((float)K.xvw) * ld2(A.mu.yz, id + 1) * (ld2(wn, id + 1) - ld2(wn, id - sy + 1));
            s4 = S2((float)K.xvw) * ld2(A.mu.yz, id) * (ld2(wn, id) - ld2(wn, id - sy));
        } else {
            s1 = S2((float)K.xwu) * ld2(A.mu.xz, id + sx) * (ld2(un, id + sx) - ld2(un, id + sx - 1));
            s2 = S2((float)K.xwu) * ld2(A.mu.xz, id) * (ld2(un, id) - ld2(un, id - 1));
            s3 = S2((float)K.xwv) * ld2(A.mu.yz, id + sy) * (ld2(vn, id + sy) - ld2(vn, id + sy - 1));
            s4 = S2((float)K.xwv) * ld2(A.mu.yz, id) * (ld2(vn, id) - ld2(vn, id - 1));
        }
        H = neg2(ct) + s1 - s2 + s3 - s4;
    }
    A.H[id] = H.v.x;
    if (live_b) A.H[id + EP_DK] = H.v.y;

    // right-hand side dt*(gamma H + rho H_old + alpha A q_old + alpha body)
    const f2 dt = S2((float)A.scal[S_DT]);
    const f2 alpha = S2((float)A.alpha);
    const f2 conv = fma2(S2((float)A.r), ld2(A.Hm, id), S2((float)A.g) * H);
    const f2 q0 = ld2(q, id);
    f2 a, b, c;
    acoef2<VAR, 0>(K, G, A.mu, id, a, b, c);
    const f2 ax = fma2(c, ld2(q, id + sx), fma2(b, q0, a * ld2(q, id - sx)));
    acoef2<VAR, 1>(K, G, A.mu, id, a, b, c);
    const f2 ay = fma2(c, ld2(q, id + sy), fma2(b, q0, a * ld2(q, id - sy)));
    acoef2<VAR, 2>(K, G, A.mu, id, a, b, c);
    const f2 az = fma2(c, ld2(q, id + 1), fma2(b, q0, a * ld2(q, id - 1)));
    const f2 diff = alpha * (ax + ay + az);
    f2 S;
    if (VAR == VC) {
        S = dt * (conv + diff);
    } else {
        const f2 iRe = S2((float)(1.0 / K.Re));
        f2 bf;
        if (VAR == VU) {
            const f2 cval = S2(0.5f) * (ld2(A.cn, id) + ld2(A.cn, id - sx));
            bf = alpha * (S2((float)K.FxRe) * cval - ld2(A.pg, id) * iRe);
        } else if (VAR == VV) {
            const f2 cval = S2(0.5f) * (ld2(A.cn, id) + ld2(A.cn, id - sy));
            bf = alpha * (S2((float)K.FyRe) * cval - ld2(A.pg, id) * iRe);
        } else {
            bf = alpha * neg2(ld2(A.pg, id) * iRe);
        }
        S = dt * (conv + diff + bf);
    }
    A.S[id] = S.v.x;
    if (live_b) A.S[id + EP_DK] = S.v.y;
}
template <int VAR>
__global__ void __launch_bounds__(128, 16) k_explicit2(Geo G, Rng R, Consts K, ExplicitArgs<float> A)
{
    k_explicit2_run<VAR>(blockIdx, gridDim, G, R, K, A);
}
template <int VAR>
struct k_explicit2_b {
    static constexpr auto run = &k_explicit2_run<VAR>;
    static constexpr int maxt = 128, minb = 16, bminb = 8;
};

// closure codes of the first/last unknown of an ADI line:
// 1 b+=a (Neumann / symmetry), 2 b-=a (reflection about a wall face),
// 3 rhs-=a*0 (Dirichlet wall face), 0 none
template <int VAR, int AXIS>
struct Closure {
    // x: c L675, u L1075, v L1231, w L1378 ; y: c L610, u L1010, v L1167,
    // w L1317 ; z: c L640, u L1039, v L1196, w L1344
    static constexpr int lo = AXIS == 0 ? (VAR <= VU ? 3 : 2)
                            : AXIS == 1 ? (VAR == VC ? 1 : VAR == VV ? 3 : 2)
                                        : (VAR == VW ? 3 : 1);
    static constexpr int hi = AXIS == 0 ? 0 : lo;
};

template <typename real>
struct XsweepArgs {
    MuPtrs<real> mu;     // mu_new
    const real* q;       // q_old
    real* qn;            // q_new (out)
    real* H;             // explicit term (outflow plane written here)
    const real* Hm;      // previous explicit term
    real* S;             // eliminated rhs from the y/z sweeps (scratch)
    real* cc;            // scratch
    const double* scal;  // dt, vbulk
    double g, r, alpha;
};

// ---------------------------------------------------------------------------
// ADI line solve along z (the contiguous axis): (1 - fac A) x = S, serial
// Thomas as tridiag_1rhs (pllcart3d.c:3511-3536; concentration L592-650,
// xmom L991-1049, ymom L1148-1206, zmom L1300-1354).  Each warp owns 32
// neighbouring lines (fixed i, consecutive j) and moves them through shared
// memory in tiles of 32 lines x ZW positions, so that every global access is
// a coalesced row segment instead of 32 lines' worth of strided ones.  Forward elimination writes c'
// to `cc` and the eliminated rhs over S, tile by tile; back substitution
// walks the tiles in reverse.  The recurrence is latency-bound (one
// dependent chain per lane), so the tiles are kept narrow (ZW = 16) to
// leave room for twice the resident warps that hide it.
// ---------------------------------------------------------------------------
constexpr int ZW = 16;

template <int VAR, typename real>
constexpr size_t adi_z_smem_bytes()
{
    // per warp: S and c' tiles [32][ZW+1], viscosity tile [32][ZW+3]
    return sizeof(real) * 4 * 32 * (2 * (ZW + 1) + (VAR == VC ? 0 : ZW + 3));
}

template <int VAR, typename real>
__device__ __forceinline__ void k_adi_z_tiled_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, MuPtrs<real> mu,
                                                     real* __restrict__ S, real* __restrict__ cc,
                                                     const double* __restrict__ scal, double alpha)
{
    constexpr int W = 32;
    extern __shared__ __align__(16) unsigned char zsm[];
    typedef real Tile[W][ZW + 1];
    typedef real MTile[W][ZW + 3];
    Tile* tS = (Tile*)zsm;
    Tile* tC = tS + 4;
    MTile* tM = (MTile*)(tC + 4);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = R.is + blockIdx.y;
    const int j0 = R.js + (blockIdx.x * 4 + warp) * W;
    if (j0 > R.je) return;  // warp-uniform
    const int nl = (R.je - j0 + 1) < W ? (R.je - j0 + 1) : W;
    const int n = R.ke - R.ks + 1;
    const real fac = (real)(0.5 * scal[S_DT] * alpha);
    constexpr int LO = Closure<VAR, 2>::lo, HI = Closure<VAR, 2>::hi;
    const real* __restrict__ mz = VAR == VU ? mu.xz : VAR == VV ? mu.yz : mu.cell;
    const int moff = VAR == VW ? -1 : 0;
    const double dz_coef = VAR == VW ? K.d2z : K.d1z;
    const long base0 = (long)i * G.sx + (long)j0 * G.sy + R.ks;
    // tile moves: two rows per warp instruction (lanes 0-15 row r, 16-31
    // row r+1).  The next tile's loads go to registers before the current
    // tile's sequential solve, so global latency overlaps the recurrence.
    constexpr int NR = W / 2;
    const int hr = lane >> 4, col = lane & (ZW - 1);
    real pS[NR], pM[NR], pE;
    // 32-bit offsets from the warp's first row (a plane of a field is far
    // below 2^31 elements)
    const int sy = (int)G.sy;
    auto fetch_fwd = [&](int k0) {
        const int nk = (n - k0) < ZW ? (n - k0) : ZW;
        const real* Sb = S + base0 + k0;
        const real* Mb = mz + base0 + k0 + moff;
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            const int r = 2 * q + hr;
            const bool ok = r < nl && col < nk;
            pS[q] = ok ? Sb[r * sy + col] : (real)0;
            if (VAR != VC) pM[q] = ok ? Mb[r * sy + col] : (real)0;
        }
        // the viscosity value one past the tile, lane = row
        if (VAR != VC) pE = lane < nl ? Mb[lane * sy + nk] : (real)0;
    };
    auto fetch_bwd = [&](int k0) {
        const int nk = (n - k0) < ZW ? (n - k0) : ZW;
        const real* Sb = S + base0 + k0;
        const real* Cb = cc + base0 + k0;
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            const int r = 2 * q + hr;
            const bool ok = r < nl && col < nk;
            pS[q] = ok ? Sb[r * sy + col] : (real)0;
            pM[q] = ok ? Cb[r * sy + col] : (real)0;
        }
    };
    real cprev = 0, rprev = 0;
    fetch_fwd(0);
    for (int k0 = 0; k0 < n; k0 += ZW) {
        const int nk = (n - k0) < ZW ? (n - k0) : ZW;
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            const int r = 2 * q + hr;
            if (r < nl && col < nk) {
                tS[warp][r][col] = pS[q];
                if (VAR != VC) tM[warp][r][col] = pM[q];
            }
        }
        if (VAR != VC && lane < nl) tM[warp][lane][nk] = pE;
        __syncwarp();
        if (k0 + ZW < n) fetch_fwd(k0 + ZW);
        if (lane < nl) {
            for (int t = 0; t < nk; ++t) {
                const int m = k0 + t;
                real a, c;
                if (VAR == VC) {
                    a = (real)K.cdz;
                    c = (real)K.cdz;
                } else {
                    a = over_h<real>((real)dz_coef * tM[warp][lane][t], K.hz, K.ihz, K.pow2);
                    c = over_h<real>((real)dz_coef * tM[warp][lane][t + 1], K.hz, K.ihz, K.pow2);
                }
                const real b = -(a + c);
                real la = -fac * a, lb = (real)1.0 - fac * b, lc = -fac * c, lr = tS[warp][lane][t];
                if (m == 0) {
                    if (LO == 1) lb += la;
                    else if (LO == 2) lb -= la;
                    else if (LO == 3) lr -= la * (real)0.0;
                }
                if (m == n - 1) {
                    if (HI == 1) lb += lc;
                    else if (HI == 2) lb -= lc;
                    else if (HI == 3) lr -= lc * (real)0.0;
                }
                real bb, cm, rm;
                if (m == 0) {
                    bb = lb;
                    thomas_div<real>(lc, lr, bb, cm, rm);
                } else {
                    bb = lb - cprev * la;
                    thomas_div<real>(lc, (lr - rprev * la), bb, cm, rm);
                }
                tC[warp][lane][t] = cm;
                tS[warp][lane][t] = rm;
                cprev = cm;
                rprev = rm;
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            const int r = 2 * q + hr;
            if (r < nl && col < nk) {
                S[base0 + k0 + r * sy + col] = tS[warp][r][col];
                cc[base0 + k0 + r * sy + col] = tC[warp][r][col];
            }
        }
        __syncwarp();
    }
    // back substitution, last tile first; x_{n-1} = r'_{n-1}.  Every tile's
    // S and c' were stored by this warp above (same lanes, same addresses).
    real xnext = rprev;
    const int last0 = ((n - 1) / ZW) * ZW;
    fetch_bwd(last0);
    for (int k0 = last0; k0 >= 0; k0 -= ZW) {
        const int nk = (n - k0) < ZW ? (n - k0) : ZW;
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            const int r = 2 * q + hr;
            if (r < nl && col < nk) {
                tS[warp][r][col] = pS[q];
                tC[warp][r][col] = pM[q];
            }
        }
        __syncwarp();
        if (k0 - ZW >= 0) fetch_bwd(k0 - ZW);
        if (lane < nl) {
            for (int t = nk - 1; t >= 0; --t) {
                const int m = k0 + t;
                if (m == n - 1) continue;
                real x = tS[warp][lane][t] - xnext * tC[warp][lane][t];
                tS[warp][lane][t] = x;
                xnext = x;
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            const int r = 2 * q + hr;
            if (r < nl && col < nk) S[base0 + k0 + r * sy + col] = tS[warp][r][col];
        }
        __syncwarp();
    }
}
template <int VAR, typename real>
__global__ void __launch_bounds__(128, 4) k_adi_z_tiled(Geo G, Rng R, Consts K, MuPtrs<real> mu,
                                                     real* __restrict__ S, real* __restrict__ cc,
                                                     const double* __restrict__ scal, double alpha)
{
    k_adi_z_tiled_run<VAR, real>(blockIdx, gridDim, G, R, K, mu, S, cc, scal, alpha);
}
template <int VAR, typename real>
struct k_adi_z_tiled_b {
    static constexpr auto run = &k_adi_z_tiled_run<VAR, real>;
    static constexpr int maxt = 128, minb = 4;
};


// ---------------------------------------------------------------------------
// The precision form's z line solve: one warp per line, the line held in
// registers (8 rows per lane) and solved by a partition method instead of
// the sequential Thomas chain.  Row 8l of each lane is a separator; the lane
// eliminates its 7 interior rows in terms of its own separator and the next
// lane's (x_e = g_e - v_e S_l - w_e S_{l+1}), the 32 separator equations
// form a tridiagonal system solved by parallel cyclic reduction over warp
// shuffles, and the interior rows follow.  S is read once and the solution
// written once (the Thomas form also writes and re-reads c' and the
// eliminated right-hand side).  Same coefficients and closures as
// k_adi_z_tiled; FP32-level agreement, not bitwise.  Lines of up to 256.
// Rows move between global memory (coalesced, row m by lane m % 32) and the
// lane that owns them (8l .. 8l+7) through a skewed shared buffer.
// ---------------------------------------------------------------------------
constexpr int ZP_MAX = 256;
__device__ __forceinline__ int zp_skew(int m) { return m + (m >> 3); }

// 1/x of the partitioned solves: FP32 approximate (<= 2 ulp; the pivots of
// these diagonally dominant systems are >= 1 in magnitude), FP64 IEEE
template <typename real>
__device__ __forceinline__ real rcp_(real x) { return (real)1 / x; }
template <>
__device__ __forceinline__ float rcp_<float>(float x) { return __fdividef(1.0f, x); }

// Partitioned solve of one line of 32 E rows held E per lane (rows
// E l .. E l + E - 1 on lane l; a of the first row and c of the last are 0;
// rows past the line are identity rows): row E l of each lane is a
// separator, the lane eliminates its E-1 interior rows in terms of its own
// separator and the next lane's (x_e = g_e - v_e S_l - w_e S_{l+1}), the 32
// separator equations are solved by parallel cyclic reduction over warp
// shuffles, then the interior rows.  FP32, diagonally dominant systems.
template <typename real, int E>
__device__ __forceinline__ void zp_solve(const real* A, const real* B, const real* C, const real* Rr, real* x,
                                         int lane)
{
    // interior rows e = 1..E-1: forward in terms of the own separator S_l
    real ch[E], rh[E], ah[E];
    {
        const real ib = rcp_<real>(B[1]);
        ch[1] = C[1] * ib;
        rh[1] = Rr[1] * ib;
        ah[1] = A[1] * ib;
    }
#pragma unroll
    for (int e = 2; e < E; ++e) {
        const real id = rcp_<real>(B[e] - A[e] * ch[e - 1]);
        ch[e] = C[e] * id;
        rh[e] = (Rr[e] - A[e] * rh[e - 1]) * id;
        ah[e] = -A[e] * ah[e - 1] * id;
    }
    // backward: x_e = g_e - v_e S_l - w_e S_{l+1}
    real g[E], v[E], w[E];
    g[E - 1] = rh[E - 1];
    v[E - 1] = ah[E - 1];
    w[E - 1] = ch[E - 1];
#pragma unroll
    for (int e = E - 2; e >= 1; --e) {
        g[e] = rh[e] - ch[e] * g[e + 1];
        v[e] = ah[e] - ch[e] * v[e + 1];
        w[e] = -ch[e] * w[e + 1];
    }
    // separator row 8l: A0 x_{8l-1} + B0 S_l + C0 x_{8l+1} = R0
    real gp = __shfl_up_sync(0xffffffffu, g[E - 1], 1);
    real vp = __shfl_up_sync(0xffffffffu, v[E - 1], 1);
    real wp = __shfl_up_sync(0xffffffffu, w[E - 1], 1);
    if (lane == 0) gp = vp = wp = (real)0;
    real al = -A[0] * vp;
    real be = B[0] - A[0] * wp - C[0] * v[1];
    real ga = -C[0] * w[1];
    real rho = Rr[0] - A[0] * gp - C[0] * g[1];
    // parallel cyclic reduction of the 32 separator equations
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        real al_m = __shfl_up_sync(0xffffffffu, al, d), be_m = __shfl_up_sync(0xffffffffu, be, d);
        real ga_m = __shfl_up_sync(0xffffffffu, ga, d), rho_m = __shfl_up_sync(0xffffffffu, rho, d);
        real al_p = __shfl_down_sync(0xffffffffu, al, d), be_p = __shfl_down_sync(0xffffffffu, be, d);
        real ga_p = __shfl_down_sync(0xffffffffu, ga, d), rho_p = __shfl_down_sync(0xffffffffu, rho, d);
        if (lane < d) {
            al_m = (real)0;
            be_m = (real)1;
            ga_m = (real)0;
            rho_m = (real)0;
        }
        if (lane + d > 31) {
            al_p = (real)0;
            be_p = (real)1;
            ga_p = (real)0;
            rho_p = (real)0;
        }
        const real k1 = al * rcp_<real>(be_m), k2 = ga * rcp_<real>(be_p);
        const real nal = -k1 * al_m, nga = -k2 * ga_p;
        be = be - k1 * ga_m - k2 * al_p;
        rho = rho - k1 * rho_m - k2 * rho_p;
        al = nal;
        ga = nga;
    }
    const real Sl = rho * rcp_<real>(be);
    real Sn = __shfl_down_sync(0xffffffffu, Sl, 1);
    if (lane == 31) Sn = (real)0;
    x[0] = Sl;
#pragma unroll
    for (int e = 1; e < E; ++e) x[e] = g[e] - v[e] * Sl - w[e] * Sn;
}

template <int VAR, typename real>
__device__ __forceinline__ void k_adi_z_part_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, MuPtrs<real> mu,
                                                    real* __restrict__ S, const double* __restrict__ scal,
                                                    double alpha)
{
    constexpr int E = ZP_MAX / 32;   // rows per lane
    constexpr int BUF = ZP_MAX + ZP_MAX / 8 + 8;
    __shared__ real bS[4][BUF];
    __shared__ real bM[4][BUF];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j = R.js + blockIdx.x * 4 + warp;
    const int i = R.is + blockIdx.y;
    if (j > R.je) return;   // warp-uniform
    const int n = R.ke - R.ks + 1;
    const real fac = (real)(0.5 * scal[S_DT] * alpha);
    constexpr int LO = Closure<VAR, 2>::lo, HI = Closure<VAR, 2>::hi;
    const real* __restrict__ mz = VAR == VU ? mu.xz : VAR == VV ? mu.yz : mu.cell;
    const int moff = VAR == VW ? -1 : 0;
    const real dzc = (real)(VAR == VW ? K.d2z : K.d1z);
    const real ihz = (real)K.ihz, cdz = (real)K.cdz;
    const long base = (long)i * G.sx + (long)j * G.sy + R.ks;
    real* sS = bS[warp];
    real* sM = bM[warp];
#pragma unroll
    for (int t = 0; t < E; ++t) {
        const int m = t * 32 + lane;
        if (m < n) sS[zp_skew(m)] = S[base + m];
        if (VAR != VC && m <= n) sM[zp_skew(m)] = mz[base + moff + m];
    }
    if (VAR != VC && lane == 0 && n == ZP_MAX) sM[zp_skew(ZP_MAX)] = mz[base + moff + ZP_MAX];
    __syncwarp();

    // this lane's rows m = 8 lane + e: a x_{m-1} + b x_m + c x_{m+1} = r
    real A[E], B[E], C[E], Rr[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int m = E * lane + e;
        if (m < n) {
            real a, c;
            if (VAR == VC) {
                a = cdz;
                c = cdz;
            } else {
                a = dzc * sM[zp_skew(m)] * ihz;
                c = dzc * sM[zp_skew(m + 1)] * ihz;
            }
            const real b = -(a + c);
            real la = -fac * a, lb = (real)1.0 - fac * b, lc = -fac * c, lr = sS[zp_skew(m)];
            if (m == 0) {
                if (LO == 1) lb += la;
                else if (LO == 2) lb -= la;
                la = (real)0;
            }
            if (m == n - 1) {
                if (HI == 1) lb += lc;
                else if (HI == 2) lb -= lc;
                lc = (real)0;
            }
            A[e] = la;
            B[e] = lb;
            C[e] = lc;
            Rr[e] = lr;
        } else {   // identity rows past the line
            A[e] = (real)0;
            B[e] = (real)1;
            C[e] = (real)0;
            Rr[e] = (real)0;
        }
    }
    real x[E];
    zp_solve<real, E>(A, B, C, Rr, x, lane);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e) sS[zp_skew(E * lane + e)] = x[e];
    __syncwarp();
#pragma unroll
    for (int t = 0; t < E; ++t) {
        const int m = t * 32 + lane;
        if (m < n) S[base + m] = sS[zp_skew(m)];
    }
}
template <int VAR, typename real>
__global__ void __launch_bounds__(128) k_adi_z_part(Geo G, Rng R, Consts K, MuPtrs<real> mu,
                                                    real* __restrict__ S, const double* __restrict__ scal,
                                                    double alpha)
{
    k_adi_z_part_run<VAR, real>(blockIdx, gridDim, G, R, K, mu, S, scal, alpha);
}
template <int VAR, typename real>
struct k_adi_z_part_b {
    static constexpr auto run = &k_adi_z_part_run<VAR, real>;
    static constexpr int maxt = 128, minb = 0;
};


// ---------------------------------------------------------------------------
// Viscosity family and offset that the implicit coefficients of VAR along
// AXIS read (A_umom/A_vmom/A_wmom, pllcart3d.c:1443-1536): a at line
// position m uses family[m + OFF], c uses family[m + OFF + 1]; the scale is
// 2/(Re h) on the variable's own axis and 1/(Re h) across.
// ---------------------------------------------------------------------------
template <int VAR, int AXIS>
struct LineCoef {
    static constexpr int fam = VAR == VC ? -1
                             : (VAR == VU && AXIS == 0) || (VAR == VV && AXIS == 1) || (VAR == VW && AXIS == 2) ? MU_CELL_
                             : (VAR == VU && AXIS == 1) || (VAR == VV && AXIS == 0) ? MU_XY_
                             : (VAR == VU && AXIS == 2) || (VAR == VW && AXIS == 0) ? MU_XZ_
                                                                                      : MU_YZ_;
    static constexpr int off = fam == MU_CELL_ ? -1 : 0;
    static constexpr bool twice = fam == MU_CELL_;
};

template <int VAR, int AXIS, typename real>
__device__ __forceinline__ const real* line_family(const MuPtrs<real>& mu)
{
    constexpr int f = LineCoef<VAR, AXIS>::fam;
    return f == MU_CELL_ ? mu.cell : f == MU_XY_ ? mu.xy : f == MU_XZ_ ? mu.xz : mu.yz;
}

// a, c of the ADI operator from two consecutive family values (same
// expressions as acoef)
template <int VAR, int AXIS, typename real>
__device__ __forceinline__ void line_ac(const Consts& K, real m0, real m1, real& a, real& c)
{
    const double h = AXIS == 0 ? K.hx : AXIS == 1 ? K.hy : K.hz;
    const double ih = AXIS == 0 ? K.ihx : AXIS == 1 ? K.ihy : K.ihz;
    if (VAR == VC) {
        a = c = (real)(AXIS == 0 ? K.cdx : AXIS == 1 ? K.cdy : K.cdz);
    } else {
        const double d = LineCoef<VAR, AXIS>::twice ? (AXIS == 0 ? K.d2x : AXIS == 1 ? K.d2y : K.d2z)
                                                     : (AXIS == 0 ? K.d1x : AXIS == 1 ? K.d1y : K.d1z);
        a = over_h<real>((real)d * m0, h, ih, K.pow2);
        c = over_h<real>((real)d * m1, h, ih, K.pow2);
    }
}

// ---------------------------------------------------------------------------
// The precision form's y line solve with the same partitioned warp solver:
// a block of 8 warps stages 32 neighbouring lines (consecutive k, coalesced
// rows of the tile) and their viscosity family through shared memory, each
// warp solves 4 of them, the block writes the solutions back in place.  Same
// coefficients and closures as k_line_pf<VAR, 1>; S read once, written once.
// ---------------------------------------------------------------------------
constexpr int YP_PITCH = ZP_MAX + ZP_MAX / 8 + 1;   // odd: conflict-free columns

template <typename real>
constexpr size_t adi_y_part_smem() { return sizeof(real) * 2 * 32 * YP_PITCH; }

template <int VAR, typename real>
__device__ __forceinline__ void k_adi_y_part_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, MuPtrs<real> mu,
                                                    real* __restrict__ S, const double* __restrict__ scal,
                                                    double alpha)
{
    constexpr int E = ZP_MAX / 32;
    extern __shared__ __align__(16) unsigned char ysm_raw[];
    real* ysm = (real*)ysm_raw;
    real* tS = ysm;                      // [32 lines][YP_PITCH]
    real* tM = ysm + 32 * YP_PITCH;
    const int i = R.is + blockIdx.y;
    const int k0 = R.ks + blockIdx.x * 32;
    const int nl = (R.ke - k0 + 1) < 32 ? (R.ke - k0 + 1) : 32;
    const int n = R.je - R.js + 1;
    const long sy = G.sy;
    const long base0 = (long)i * G.sx + (long)R.js * sy + k0;
    constexpr int OFF = LineCoef<VAR, 1>::off;
    const real* __restrict__ fam = VAR == VC ? nullptr : line_family<VAR, 1, real>(mu);
    const real dy = (real)(LineCoef<VAR, 1>::twice ? K.d2y : K.d1y);
    const real ihy = (real)K.ihy, cdy = (real)K.cdy;
    const real fac = (real)(0.5 * scal[S_DT] * alpha);
    constexpr int LO = Closure<VAR, 1>::lo, HI = Closure<VAR, 1>::hi;
    // tile loads: thread (kl, row group m0) moves rows m0, m0 + 8, ...;
    // unrolled so that many rows' loads are in flight at once
    const int tkl = threadIdx.x & 31, tm0 = threadIdx.x >> 5;
#pragma unroll 11
    for (int t = 0; t < ZP_MAX / 8 + 1; ++t) {
        const int m = tm0 + 8 * t;
        if (tkl < nl && m <= n) {
            if (m < n) tS[tkl * YP_PITCH + zp_skew(m)] = S[base0 + (long)m * sy + tkl];
            if (VAR != VC) tM[tkl * YP_PITCH + zp_skew(m)] = fam[base0 + (long)(m + OFF) * sy + tkl];
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int kl = warp; kl < nl; kl += 8) {
        const real* ls = tS + kl * YP_PITCH;
        const real* lm = tM + kl * YP_PITCH;
        real A[E], B[E], C[E], Rr[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int m = E * lane + e;
            if (m < n) {
                real a, c;
                if (VAR == VC) {
                    a = cdy;
                    c = cdy;
                } else {
                    a = dy * lm[zp_skew(m)] * ihy;
                    c = dy * lm[zp_skew(m + 1)] * ihy;
                }
                const real b = -(a + c);
                real la = -fac * a, lb = (real)1.0 - fac * b, lc = -fac * c;
                if (m == 0) {
                    if (LO == 1) lb += la;
                    else if (LO == 2) lb -= la;
                    la = (real)0;
                }
                if (m == n - 1) {
                    if (HI == 1) lb += lc;
                    else if (HI == 2) lb -= lc;
                    lc = (real)0;
                }
                A[e] = la;
                B[e] = lb;
                C[e] = lc;
                Rr[e] = ls[zp_skew(m)];
            } else {
                A[e] = (real)0;
                B[e] = (real)1;
                C[e] = (real)0;
                Rr[e] = (real)0;
            }
        }
        real x[E];
        zp_solve<real, E>(A, B, C, Rr, x, lane);
        __syncwarp();
#pragma unroll
        for (int e = 0; e < E; ++e) tS[kl * YP_PITCH + zp_skew(E * lane + e)] = x[e];
    }
    __syncthreads();
#pragma unroll 8
    for (int t = 0; t < ZP_MAX / 8; ++t) {
        const int m = tm0 + 8 * t;
        if (tkl < nl && m < n) S[base0 + (long)m * sy + tkl] = tS[tkl * YP_PITCH + zp_skew(m)];
    }
}
template <int VAR, typename real>
__global__ void __launch_bounds__(256) k_adi_y_part(Geo G, Rng R, Consts K, MuPtrs<real> mu,
                                                    real* __restrict__ S, const double* __restrict__ scal,
                                                    double alpha)
{
    k_adi_y_part_run<VAR, real>(blockIdx, gridDim, G, R, K, mu, S, scal, alpha);
}
template <int VAR, typename real>
struct k_adi_y_part_b {
    static constexpr auto run = &k_adi_y_part_run<VAR, real>;
    static constexpr int maxt = 256, minb = 0;
};

// ---------------------------------------------------------------------------
// Line solves along a strided axis (AXIS 0: x, lines (j,k); AXIS 1: y,
// lines (i,k)), one thread per line, adjacent threads on adjacent k so every
// access is coalesced.  The loads of PF line positions ahead (rhs and one
// viscosity value per position) are issued before the dependent Thomas
// recurrence consumes them, so the sweep streams instead of waiting one
// memory latency per position.  AXIS 1 is tridiag_1rhs (pllcart3d.c:3511);
// AXIS 0 is pll_tridiag's one-rank form (pll_tridiag.c:21-47, 96-110) with
// the convective outflow (e.g. pllcart3d.c:677-683), q_new = q_old + delta
// and, for c, the Neumann ghosts of pllcart3d.c:700-712.
// ---------------------------------------------------------------------------
template <int VAR, int AXIS, typename real>
__device__ __forceinline__ void k_line_pf_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, XsweepArgs<real> A)
{
    constexpr int PF = 8;
    const int k = R.ks + blockIdx.x * blockDim.x + threadIdx.x;
    const int o = blockIdx.y;  // j (AXIS 0) or i (AXIS 1) offset
    if (k > R.ke) return;
    const long st = AXIS == 0 ? G.sx : G.sy;
    const int n = AXIS == 0 ? R.ie - R.is + 1 : R.je - R.js + 1;
    const long base = AXIS == 0 ? (long)R.is * G.sx + (long)(R.js + o) * G.sy + k
                                : (long)(R.is + o) * G.sx + (long)R.js * G.sy + k;
    const real dt = (real)A.scal[S_DT];
    const real fac = (real)(0.5 * A.scal[S_DT] * A.alpha);
    constexpr int LO = Closure<VAR, AXIS>::lo, HI = Closure<VAR, AXIS>::hi;
    constexpr int OFF = LineCoef<VAR, AXIS>::off;
    const real* __restrict__ fam = VAR == VC ? nullptr : line_family<VAR, AXIS, real>(A.mu);
    real* __restrict__ S = A.S;
    real* __restrict__ cc = A.cc;

    real boun = 0;
    if (AXIS == 0) {
        const long rb = base + (long)n * st;
        real Hb = -(real)A.scal[S_VBULK] * (A.q[rb] - A.q[rb - st]);
        Hb = over_h<real>(Hb, K.hx, K.ihx, K.pow2);
        A.H[rb] = Hb;
        boun = rk_step<real>(dt, (real)A.g, Hb, (real)A.r, A.Hm[rb]);
        A.qn[rb] = A.q[rb] + boun;
    }

    // forward elimination
    real cprev = 0, rprev = 0;
    real mlast = VAR == VC ? (real)0 : fam[base + (long)OFF * st];
    real sv[PF], mv[PF];
#pragma unroll
    for (int t = 0; t < PF; ++t) {
        sv[t] = t < n ? S[base + (long)t * st] : (real)0;
        if (VAR != VC) mv[t] = t < n ? fam[base + (long)(t + OFF + 1) * st] : (real)0;
    }
    for (int m0 = 0; m0 < n; m0 += PF) {
        real sn[PF], mn[PF];
#pragma unroll
        for (int t = 0; t < PF; ++t) {
            const int m = m0 + PF + t;
            sn[t] = m < n ? S[base + (long)m * st] : (real)0;
            if (VAR != VC) mn[t] = m < n ? fam[base + (long)(m + OFF + 1) * st] : (real)0;
        }
#pragma unroll
        for (int t = 0; t < PF; ++t) {
            const int m = m0 + t;
            if (m < n) {
                real a, c;
                line_ac<VAR, AXIS, real>(K, mlast, VAR == VC ? (real)0 : mv[t], a, c);
                if (VAR != VC) mlast = mv[t];
                const real b = -(a + c);
                real la = -fac * a, lb = (real)1.0 - fac * b, lc = -fac * c, lr = sv[t];
                if (m == 0) {
                    if (LO == 1) lb += la;
                    else if (LO == 2) lb -= la;
                    else if (LO == 3) lr -= la * (real)0.0;
                }
                if (m == n - 1) {
                    if (AXIS == 0) lr -= lc * boun;
                    else if (HI == 1) lb += lc;
                    else if (HI == 2) lb -= lc;
                    else if (HI == 3) lr -= lc * (real)0.0;
                }
                real cm, rm;
                if (AXIS == 0) {
                    if (m == 0) {
                        lb = lb - (real)0.0 * la;
                        thomas_div<real>(lc, (lr - (real)0.0 * la), lb, cm, rm);
                    } else {
                        lb = (lb - cprev * la);
                        thomas_div<real>(lc, (lr - rprev * la), lb, cm, rm);
                    }
                } else {
                    if (m == 0) {
                        thomas_div<real>(lc, lr, lb, cm, rm);
                    } else {
                        const real bb = lb - cprev * la;
                        thomas_div<real>(lc, (lr - rprev * la), bb, cm, rm);
                    }
                }
                const long id = base + (long)m * st;
                cc[id] = cm;
                S[id] = rm;
                cprev = cm;
                rprev = rm;
            }
        }
#pragma unroll
        for (int t = 0; t < PF; ++t) {
            sv[t] = sn[t];
            if (VAR != VC) mv[t] = mn[t];
        }
    }

    // q_new at line position id; for c also its Neumann ghosts in y
    // (pllcart3d.c:700-705) then z (L707-712), written as the value is
    // produced.  The z copies run over j in [js-1, je+1] in the reference,
    // so its corners copy the y ghosts, which equal this line's value.
    const int jl = R.js + o;
    const bool jlo = AXIS == 0 && VAR == VC && jl == R.js, jhi = AXIS == 0 && VAR == VC && jl == R.je;
    const bool klo = AXIS == 0 && VAR == VC && k == R.ks, khi = AXIS == 0 && VAR == VC && k == R.ke;
    const bool edge = jlo | jhi | klo | khi;
    auto put = [&](long id, real v) {
        A.qn[id] = v;
        if (edge) {
            const long sy = G.sy;
            if (jlo) A.qn[id - sy] = v;
            if (jhi) A.qn[id + sy] = v;
            if (klo) {
                A.qn[id - 1] = v;
                if (jlo) A.qn[id - sy - 1] = v;
                if (jhi) A.qn[id + sy - 1] = v;
            }
            if (khi) {
                A.qn[id + 1] = v;
                if (jlo) A.qn[id - sy + 1] = v;
                if (jhi) A.qn[id + sy + 1] = v;
            }
        }
    };

    // back substitution, x_{n-1} = r'_{n-1} (pll form: minus c' * 0)
    real xnext = AXIS == 0 ? rprev - cprev * (real)0.0 : rprev;
    if (AXIS == 0) {
        const long id = base + (long)(n - 1) * st;
        put(id, A.q[id] + xnext);
    }
    // positions n-2 .. 0 in chunks of PF, loads of the next chunk first
    real rv[PF], cv[PF], qv[PF];
    int mtop = n - 2;
#pragma unroll
    for (int t = 0; t < PF; ++t) {
        const int m = mtop - t;
        const long id = base + (long)m * st;
        rv[t] = m >= 0 ? S[id] : (real)0;
        cv[t] = m >= 0 ? cc[id] : (real)0;
        if (AXIS == 0) qv[t] = m >= 0 ? A.q[id] : (real)0;
    }
    for (; mtop >= 0; mtop -= PF) {
        real rn[PF], cn2[PF], qn2[PF];
#pragma unroll
        for (int t = 0; t < PF; ++t) {
            const int m = mtop - PF - t;
            const long id = base + (long)m * st;
            rn[t] = m >= 0 ? S[id] : (real)0;
            cn2[t] = m >= 0 ? cc[id] : (real)0;
            if (AXIS == 0) qn2[t] = m >= 0 ? A.q[id] : (real)0;
        }
#pragma unroll
        for (int t = 0; t < PF; ++t) {
            const int m = mtop - t;
            if (m >= 0) {
                const long id = base + (long)m * st;
                real x = AXIS == 0 ? rv[t] - cv[t] * xnext : rv[t] - xnext * cv[t];
                if (AXIS == 0) put(id, qv[t] + x);
                else S[id] = x;
                xnext = x;
            }
        }
#pragma unroll
        for (int t = 0; t < PF; ++t) {
            rv[t] = rn[t];
            cv[t] = cn2[t];
            if (AXIS == 0) qv[t] = qn2[t];
        }
    }

}
template <int VAR, int AXIS, typename real>
__global__ void __launch_bounds__(128) k_line_pf(Geo G, Rng R, Consts K, XsweepArgs<real> A)
{
    k_line_pf_run<VAR, AXIS, real>(blockIdx, gridDim, G, R, K, A);
}
template <int VAR, int AXIS, typename real>
struct k_line_pf_b {
    static constexpr auto run = &k_line_pf_run<VAR, AXIS, real>;
    static constexpr int maxt = 128, minb = 0;
};

// ---------------------------------------------------------------------------
// The precision form's line solve along a strided axis (x or y) by a
// partition method: a block owns 32 neighbouring lines (lane = line, adjacent
// k, so every row access is one coalesced 128-byte transaction) and cuts each
// line into P segments of RS rows, one warp per segment.  A thread keeps
// its segment's right-hand side in registers; its viscosity rows (momentum)
// and, for the x sweep, its q_old rows are copied into shared memory by
// cp.async, each thread copying and later reading only its own rows.  The
// thread eliminates the interior rows in terms of the segment's first row
// (its separator) and the next segment's, the P separator equations of
// every line are solved by one thread per line through shared memory, and
// each thread finishes its rows with the separators known.  Every input is
// read once from HBM and every output written once (the sequential sweep
// also writes and re-reads c' and the eliminated rhs).  Same coefficients
// and closures as k_line_pf (x: convective outflow, q_new = q_old + delta,
// concentration's Neumann ghosts; y: in place into S); FP32-level agreement
// with the sequential sweep, not bitwise.
// ---------------------------------------------------------------------------

// dynamic shared memory of k_line_seg: the viscosity family's rows (RS + 1
// per thread, momentum) then the x sweep's q_old rows (RS per thread)
template <int VAR, int AXIS, int P, int RS, typename real = float>
constexpr size_t line_seg_smem()
{
    return sizeof(real) * 32 * P * ((VAR != VC ? RS + 1 : 0) + (AXIS == 0 ? RS : 0));
}

// one element global -> shared by cp.async (4 or 8 bytes)
template <typename real>
__device__ __forceinline__ void ls_cp_async(real* dst, const real* src)
{
    if (sizeof(real) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                     "l"(src)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                     "l"(src)
                     : "memory");
}

// an optimisation barrier on x: later reads cannot reuse values computed
// from it before (keeps each sweep recomputing its row coefficients instead
// of holding four per row in registers; a "memory" clobber does the same
// for the shared-memory rows)
__device__ __forceinline__ void ls_fresh(float& x) { asm volatile("" : "+f"(x)); }
__device__ __forceinline__ void ls_fresh(double& x) { asm volatile("" : "+d"(x)); }

// FULL: the line has P * RS rows; else P * RS - 1 and the last
// segment's last row is an identity row (its loads read the row past the
// line, which the host checks lies inside the padded box)
template <int VAR, int AXIS, int P, int RS, bool FULL, typename real = float>
__device__ __forceinline__ void k_line_seg_run(const uint3 blockIdx, const dim3 gridDim,
    Geo G, Rng R, Consts K, XsweepArgs<real> A)
{
    __shared__ real eq[4][P][32];       // separator equations
    __shared__ real tail[3][P][32];     // last interior row of each segment
    __shared__ real sep[P + 1][32];     // separator values
    extern __shared__ __align__(16) unsigned char ls_raw[];
    real* ls_dyn = (real*)ls_raw;       // [row][thread] tiles: viscosity, then q_old (x)
    constexpr int LO = Closure<VAR, AXIS>::lo, HI = Closure<VAR, AXIS>::hi;
    constexpr int OFF = LineCoef<VAR, AXIS>::off;
    constexpr int TS = 32 * P;
    const int lane = threadIdx.x & 31, l = threadIdx.x >> 5;
    const int k = R.ks + blockIdx.x * 32 + lane;
    const int o = blockIdx.y;   // j (AXIS 0) or i (AXIS 1) offset
    const bool live = k <= R.ke;
    const bool last_seg = l == P - 1;
    constexpr int n = FULL ? P * RS : P * RS - 1;
    // offsets fit in 32 bits (the host checks the field size)
    const int st = AXIS == 0 ? (int)G.sx : (int)G.sy;
    const long base = AXIS == 0 ? (long)R.is * G.sx + (long)(R.js + o) * G.sy + k
                                : (long)(R.is + o) * G.sx + (long)R.js * G.sy + k;
    const long seg = base + (long)(l * RS) * st;
    const real dt = (real)A.scal[S_DT];
    const real fac = (real)(0.5 * A.scal[S_DT] * A.alpha);
    const real* __restrict__ fam = VAR == VC ? nullptr : line_family<VAR, AXIS, real>(A.mu);
    real* __restrict__ S = A.S;
    // this thread's row e of the tiles: mym[e * TS], myq[e * TS]
    real* mym = ls_dyn + threadIdx.x;
    real* myq = ls_dyn + (VAR != VC ? (RS + 1) * TS : 0) + threadIdx.x;

    if (VAR != VC) {
        if (live) {
            const real* mp = fam + seg + OFF * st;
#pragma unroll
            for (int e = 0; e <= RS; ++e) ls_cp_async<real>(mym + e * TS, mp + e * st);
        } else {
#pragma unroll
            for (int e = 0; e <= RS; ++e) mym[e * TS] = (real)0;
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    if (AXIS == 0 && live) {
#pragma unroll
        for (int e = 0; e < RS; ++e) ls_cp_async<real>(myq + e * TS, A.q + seg + e * st);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    real rS[RS];
    {
        const real* sp = S + seg;
#pragma unroll
        for (int e = 0; e < RS; ++e) rS[e] = live ? sp[e * st] : (real)0;
    }

    // convective outflow value (x): the thread that owns the line's last row
    real boun = (real)0;
    if (AXIS == 0 && live && last_seg) {
        const long rb = base + (long)n * st;
        real Hb = -(real)A.scal[S_VBULK] * (A.q[rb] - A.q[rb - st]);
        Hb = over_h<real>(Hb, K.hx, K.ihx, K.pow2);
        A.H[rb] = Hb;
        boun = rk_step<real>(dt, (real)A.g, Hb, (real)A.r, A.Hm[rb]);
        A.qn[rb] = A.q[rb] + boun;
    }
    if (VAR != VC) {
        // the viscosity rows have landed (the q rows may still be in flight)
        if (AXIS == 0 && live) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }

    // row e of this segment: (la, lb, lc, lr) with the line's closures; la of
    // the line's first row and lc of its last are dropped (the sequential
    // sweep multiplies them by zero)
    auto row = [&](int e, real& la, real& lb, real& lc, real& lr) {
        if (!FULL && last_seg && e == RS - 1) {
            la = (real)0;
            lb = (real)1;
            lc = (real)0;
            lr = (real)0;
            return;
        }
        real a, c;
        line_ac<VAR, AXIS, real>(K, VAR == VC ? (real)0 : mym[e * TS], VAR == VC ? (real)0 : mym[(e + 1) * TS], a, c);
        const real b = -(a + c);
        la = -fac * a;
        lb = (real)1 - fac * b;
        lc = -fac * c;
        lr = rS[e];
        if (e == 0 && l == 0) {
            if (LO == 1) lb += la;
            else if (LO == 2) lb -= la;
            la = (real)0;
        }
        if (last_seg && e == (FULL ? RS - 1 : RS - 2)) {
            if (AXIS == 0) lr -= lc * boun;
            else if (HI == 1) lb += lc;
            else if (HI == 2) lb -= lc;
            lc = (real)0;
        }
    };
    auto fresh = [&]() {
#pragma unroll
        for (int e = 0; e < RS; ++e) ls_fresh(rS[e]);
        asm volatile("" ::: "memory");
    };

    // interior rows top-down: x_e = rh - ah S_l - ch x_{e+1}; at the last
    // interior row x_{e+1} is the next separator
    real gL, vL, wL;
    {
        real la, lb, lc, lr;
        row(1, la, lb, lc, lr);
        real ib = rcp_<real>(lb);
        real ch = lc * ib, rh = lr * ib, ah = la * ib;
#pragma unroll
        for (int e = 2; e < RS; ++e) {
            row(e, la, lb, lc, lr);
            ib = rcp_<real>(lb - la * ch);
            rh = (lr - la * rh) * ib;
            ah = -la * ah * ib;
            ch = lc * ib;
        }
        gL = rh;
        vL = ah;
        wL = ch;
    }
    fresh();
    // bottom-up: x_e = rb - ab S_l - cb S_{l+1} down to the first interior row
    real g1, v1, w1;
    {
        real la, lb, lc, lr;
        row(RS - 1, la, lb, lc, lr);
        real ib = rcp_<real>(lb);
        real rb = lr * ib, cb = lc * ib, ab = la * ib;
#pragma unroll
        for (int e = RS - 2; e >= 1; --e) {
            row(e, la, lb, lc, lr);
            ib = rcp_<real>(lb - lc * ab);
            rb = (lr - lc * rb) * ib;
            cb = -lc * cb * ib;
            ab = la * ib;
        }
        g1 = rb;
        v1 = ab;
        w1 = cb;
    }
    fresh();
    tail[0][l][lane] = gL;
    tail[1][l][lane] = vL;
    tail[2][l][lane] = wL;
    __syncthreads();
    {
        // separator row: a0 x_{-1} + b0 S_l + c0 x_1 = r0 with x_{-1} the
        // previous segment's last interior row
        real a0, b0, c0, r0;
        row(0, a0, b0, c0, r0);
        real gp = (real)0, vp = (real)0, wp = (real)0;
        if (l > 0) {
            gp = tail[0][l - 1][lane];
            vp = tail[1][l - 1][lane];
            wp = tail[2][l - 1][lane];
        }
        eq[0][l][lane] = -a0 * vp;
        eq[1][l][lane] = b0 - a0 * wp - c0 * v1;
        eq[2][l][lane] = -c0 * w1;
        eq[3][l][lane] = r0 - a0 * gp - c0 * g1;
    }
    __syncthreads();
    if (l == 0) {
        // the P separator equations of this lane's line (Thomas); c' and
        // the eliminated rhs replace gamma and rho in place
        real ib = rcp_<real>(eq[1][0][lane]);
        real cp = eq[2][0][lane] * ib, rp = eq[3][0][lane] * ib;
        eq[2][0][lane] = cp;
        eq[3][0][lane] = rp;
#pragma unroll
        for (int t = 1; t < P; ++t) {
            const real al = eq[0][t][lane];
            ib = rcp_<real>(eq[1][t][lane] - al * cp);
            cp = eq[2][t][lane] * ib;
            rp = (eq[3][t][lane] - al * rp) * ib;
            eq[2][t][lane] = cp;
            eq[3][t][lane] = rp;
        }
        real x = rp;
        sep[P - 1][lane] = x;
        sep[P][lane] = (real)0;
#pragma unroll
        for (int t = P - 2; t >= 0; --t) {
            x = eq[3][t][lane] - eq[2][t][lane] * x;
            sep[t][lane] = x;
        }
    }
    __syncthreads();
    if (!live) return;
    const real Sl = sep[l][lane], Sn = sep[l + 1][lane];
    fresh();

    // interior rows with both separators known: Thomas with x_0 = S_l and
    // x_RS = S_{l+1}; c' in cq, the eliminated rhs replaces rS
    real cq[RS];
    {
        real la, lb, lc, lr;
        row(1, la, lb, lc, lr);
        real ib = rcp_<real>(lb);
        cq[1] = lc * ib;
        rS[1] = (lr - la * Sl) * ib;
#pragma unroll
        for (int e = 2; e < RS; ++e) {
            row(e, la, lb, lc, lr);
            ib = rcp_<real>(lb - la * cq[e - 1]);
            cq[e] = lc * ib;
            rS[e] = (lr - la * rS[e - 1]) * ib;
        }
    }
    if (AXIS == 0) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    // q_new (x; for c also its Neumann ghosts in y then z, as k_line_pf) or
    // the solution in place (y)
    const int jl = R.js + o;
    const bool jlo = AXIS == 0 && VAR == VC && jl == R.js, jhi = AXIS == 0 && VAR == VC && jl == R.je;
    const bool klo = AXIS == 0 && VAR == VC && k == R.ks, khi = AXIS == 0 && VAR == VC && k == R.ke;
    const bool edge = jlo | jhi | klo | khi;
    auto put = [&](int e, real x) {
        if (!FULL && last_seg && e == RS - 1) return;
        const long id = seg + e * st;
        if (AXIS != 0) {
            S[id] = x;
            return;
        }
        const real v = myq[e * TS] + x;
        A.qn[id] = v;
        if (edge) {
            const long sy = G.sy;
            if (jlo) A.qn[id - sy] = v;
            if (jhi) A.qn[id + sy] = v;
            if (klo) {
                A.qn[id - 1] = v;
                if (jlo) A.qn[id - sy - 1] = v;
                if (jhi) A.qn[id + sy - 1] = v;
            }
            if (khi) {
                A.qn[id + 1] = v;
                if (jlo) A.qn[id - sy + 1] = v;
                if (jhi) A.qn[id + sy + 1] = v;
            }
        }
    };
    real x = Sn;
#pragma unroll
    for (int e = RS - 1; e >= 1; --e) {
        x = rS[e] - cq[e] * x;
        put(e, x);
    }
    put(0, Sl);
}
template <int VAR, int AXIS, int P, int RS, bool FULL, typename real = float>
__global__ void __launch_bounds__(32 * P, (RS <= 16 && sizeof(real) == 4) ? 2 : 1)
    k_line_seg(Geo G, Rng R, Consts K, XsweepArgs<real> A)
{
    k_line_seg_run<VAR, AXIS, P, RS, FULL, real>(blockIdx, gridDim, G, R, K, A);
}
template <int VAR, int AXIS, int P, int RS, bool FULL, typename real = float>
struct k_line_seg_b {
    static constexpr auto run = &k_line_seg_run<VAR, AXIS, P, RS, FULL, real>;
    static constexpr int maxt = 32 * P, minb = (RS <= 16 && sizeof(real) == 4) ? 2 : 1;
};

}  // namespace
}  // namespace pll
