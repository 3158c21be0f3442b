// Explicit operator + ADI right-hand side (Hc_op/Hu_op/Hv_op/Hw_op,
// pllcart3d.c:1539-1980, with the source assembly of concentration / xmom /
// ymom / zmom, L573-590, L970-989, L1127-1146, L1280-1298) as a
// plane-marching kernel with TMA-staged shared-memory tiles.
//
// A block owns a tile of XT_TJ rows (j) x XT_TK cells (k) and walks XT_NI
// planes along x.  Every plane's tiles arrive by cp.async.bulk.tensor (one
// thread issues them; an mbarrier per ring slot counts the bytes): q with a
// +-3 halo in j and k (the WENO5 stencils along y and z), and, with a +-1
// halo, each field the variable reads at a j or k offset (velocities,
// viscosity edges, c).  A ring of XT_NS plane slots keeps planes i-1, i, i+1
// resident while plane i+2 is in flight.  Values read only along x at the
// thread's own (j, k) -- the x WENO5 window q(i-3 .. i+3), the x-face
// viscosity and velocity, c, pg, H_old -- stay in registers, one plain
// coalesced load per plane.  Every formula, closure and the stale-D2 hazard
// are k_explicit's; only where each operand comes from differs (results agree
// to rounding with the same arithmetic type and contraction flags).
// TMA boxes start on 16-byte boundaries: the k tiles start at k0 = 1 + 32 b,
// so the +-1 box starts at k0-1 (a multiple of 32 elements) and the q box at
// k0-3 (FP64: a multiple of 2) or k0-5 (FP32: a multiple of 4).  No
// multicast.  Every mbarrier wait is bounded; a wait that runs out sets
// ST_TIMEOUT, and the issuing thread drains its copies before the block ends.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "step_kernels.cuh"

namespace pll {
namespace {

constexpr int XT_TK = 32;   // k cells per tile (one warp across)
constexpr int XT_TJ = 8;    // j rows per tile (one warp each)
constexpr int XT_NS = 4;    // plane slots of the ring
constexpr int XT_NI = 32;   // planes per block
constexpr int XT_THREADS = XT_TK * XT_TJ;
constexpr long long XT_WAIT_CYCLES = 2000000000LL;   // ~1 s of SM clock

// fields staged with a +-1 halo, per variable (the ones read at a j or k
// offset besides q); order fixes the slot layout
//   VC: v, w            VU: v, w, mu_xy, mu_xz
//   VV: u, w, mu_yz, mu_cell, c_new            VW: u, v, mu_yz, mu_cell
template <int VAR>
struct XtSet {
    static constexpr int NA = VAR == VC ? 2 : VAR == VV ? 5 : 4;
};

template <typename real>
struct XtGeom {
    static constexpr int KB1 = sizeof(real) == 8 ? XT_TK + 2 : XT_TK + 4;   // +-1 box width (16-byte multiple)
    static constexpr int JB1 = XT_TJ + 2;
    static constexpr int H3 = sizeof(real) == 8 ? 3 : 5;                   // q box starts at k0 - H3
    static constexpr int KB3 = sizeof(real) == 8 ? XT_TK + 6 : XT_TK + 8;
    static constexpr int JB3 = XT_TJ + 6;
    static constexpr int T1 = ((JB1 * KB1 * (int)sizeof(real)) + 127) / 128 * 128;
    static constexpr int T3 = ((JB3 * KB3 * (int)sizeof(real)) + 127) / 128 * 128;
};

template <typename real, int VAR>
struct XtSmem {
    static constexpr int NA = XtSet<VAR>::NA;
    static constexpr int SLOT = NA * XtGeom<real>::T1 + XtGeom<real>::T3;
    static constexpr int BAR_OFF = XT_NS * SLOT;
    static constexpr int TOTAL = BAR_OFF + 64;
    static constexpr int DYN = TOTAL + 128;   // slack for 128-byte alignment
};

// the tensor maps of one launch: q (+-3 halo box) and the +-1 fields
struct XtMaps {
    CUtensorMap q;
    CUtensorMap a[5];
};

__device__ __forceinline__ uint32_t xt_saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void xt_tma_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];\n" ::"r"(xt_saddr(dst)),
        "l"((uint64_t)map), "r"(xt_saddr(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ bool xt_try_wait(uint64_t* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(xt_saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for the completion of phase `parity`
__device__ __noinline__ bool xt_wait(uint64_t* b, uint32_t parity)
{
    if (xt_try_wait(b, parity)) return true;
    const long long t0 = clock64();
    while (!xt_try_wait(b, parity))
        if (clock64() - t0 > XT_WAIT_CYCLES) return false;
    return true;
}

// upwind derivative along one axis from the 7 values q(m-3 .. m+3) of the
// line (v[3] is the point itself), the ENO-2 closure on the first and last
// two points of the range (stale-D2 values from global memory), WENO5
// elsewhere -- upwind_deriv's arithmetic
template <int AXIS, typename real>
__device__ __forceinline__ real xt_upwind(const real* v, const real* __restrict__ qg, const Geo& G, const Rng& R,
                                          const Consts& K, int m, real vv)
{
    const int s = AXIS == 0 ? R.is : AXIS == 1 ? R.js : R.ks;
    const int e = AXIS == 0 ? R.ie : AXIS == 1 ? R.je : R.ke;
    const double h = AXIS == 0 ? K.hx : AXIS == 1 ? K.hy : K.hz;
    const double ih = AXIS == 0 ? K.ihx : AXIS == 1 ? K.ihy : K.ihz;
    const double i2h = AXIS == 0 ? K.i2hx : AXIS == 1 ? K.i2hy : K.i2hz;
    const int sign = (vv >= (real)0) ? 1 : -1;
    if ((m <= s + 1) | (m >= e - 1)) {
        const bool up = sign == 1;
        const int kk = up ? m - 1 : m;
        // q(kk-1), q(kk), q(kk+1), q(kk+2): v[1..4] upwind from the left,
        // v[2..5] from the right (selected, so that v stays in registers)
        const real wm = up ? v[1] : v[2], w0 = up ? v[2] : v[3], w1 = up ? v[3] : v[4], w2 = up ? v[4] : v[5];
        real d1k = over_h<real>(w1 - w0, h, ih, K.pow2);
        real d2a, d2b;
        if (kk >= s) {
            real d1m = over_h<real>(w0 - wm, h, ih, K.pow2);
            d2a = over_2h<real>(d1k - d1m, h, i2h, K.pow2);
        } else {
            d2a = stale_d2<real>(qg, G, R, K, AXIS, kk);
        }
        if (kk + 1 <= e) {
            real d1p = over_h<real>(w2 - w1, h, ih, K.pow2);
            d2b = over_2h<real>(d1p - d1k, h, i2h, K.pow2);
        } else {
            d2b = stale_d2<real>(qg, G, R, K, AXIS, kk + 1);
        }
        real d2v = (fabs(d2a) <= fabs(d2b)) ? d2a : d2b;
        return d1k + d2v * (real)h * (real)sign;
    }
    real d[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) d[t] = over_h<real>(v[t + 1] - v[t], h, ih, K.pow2);
    const bool up = sign == 1;
    return weno5<real>(up ? d[0] : d[5], up ? d[1] : d[4], up ? d[2] : d[3], up ? d[3] : d[2], up ? d[4] : d[1]);
}

template <int VAR, typename real>
__global__ void __launch_bounds__(XT_THREADS) k_explicit_tma(const __grid_constant__ XtMaps maps, Geo G, Rng R,
                                                             Consts K, ExplicitArgs<real> A, int* status)
{
    using GM = XtGeom<real>;
    using SM = XtSmem<real, VAR>;
    constexpr int NA = XtSet<VAR>::NA;
    constexpr int KB1 = GM::KB1, KB3 = GM::KB3;
    extern __shared__ unsigned char xt_raw[];
    unsigned char* sm = (unsigned char*)(((uintptr_t)xt_raw + 127) & ~(uintptr_t)127);
    uint64_t* bar = (uint64_t*)(sm + SM::BAR_OFF);
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    const int k0 = 1 + blockIdx.x * XT_TK;
    const int j0 = R.js + blockIdx.y * XT_TJ;
    const int i0 = R.is + blockIdx.z * XT_NI;
    const int i1 = min(i0 + XT_NI - 1, R.ie);
    const int k = k0 + tx, j = j0 + ty;
    const bool live = k >= R.ks && k <= R.ke && j <= R.je;
    const long sx = G.sx, sy = G.sy;
    constexpr uint32_t STAGE_BYTES = (uint32_t)(NA * GM::JB1 * GM::KB1 + GM::JB3 * GM::KB3) * sizeof(real);

    auto slot_of = [&](int p) { return (p - (i0 - 1)) % XT_NS; };
    auto parity_of = [&](int p) { return (uint32_t)(((p - (i0 - 1)) / XT_NS) & 1); };
    auto tile1 = [&](int p, int a) { return (real*)(sm + slot_of(p) * SM::SLOT + a * GM::T1); };
    auto tile3 = [&](int p) { return (real*)(sm + slot_of(p) * SM::SLOT + NA * GM::T1); };
    auto issue = [&](int p) {   // plane p of every staged field into its slot
        uint64_t* b = &bar[slot_of(p)];
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(xt_saddr(b)),
                     "r"(STAGE_BYTES)
                     : "memory");
#pragma unroll
        for (int a = 0; a < NA; ++a) xt_tma_3d(tile1(p, a), &maps.a[a], b, k0 - 1, j0 - 1, p);
        xt_tma_3d(tile3(p), &maps.q, b, k0 - GM::H3, j0 - 3, p);
    };

    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < XT_NS; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(xt_saddr(&bar[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        issue(i0 - 1);
        issue(i0);
        issue(i0 + 1);
    }
    __syncthreads();

    // register windows along x at (j, k)
    const long col = (long)j * sy + k;
    const real* __restrict__ q = A.q;
    real qx[7];
#pragma unroll
    for (int t = 0; t < 7; ++t) qx[t] = live ? q[(long)(i0 - 3 + t) * sx + col] : (real)0;
    real xa0 = 0, xa1 = 0, xb0 = 0, xb1 = 0;   // VC: u(i), u(i+1); VU: mu_cell(i-1), (i), c(i-1), c(i);
                                               // VV: mu_xy(i), (i+1); VW: mu_xz(i), (i+1)
    const real* __restrict__ xa = VAR == VC ? A.un : VAR == VU ? A.mu.cell : VAR == VV ? A.mu.xy : A.mu.xz;
    if (live) {
        if (VAR == VU) {
            xa0 = xa[(long)(i0 - 1) * sx + col];
            xa1 = xa[(long)i0 * sx + col];
            xb0 = A.cn[(long)(i0 - 1) * sx + col];
            xb1 = A.cn[(long)i0 * sx + col];
        } else {
            xa0 = xa[(long)i0 * sx + col];
            xa1 = xa[(long)(i0 + 1) * sx + col];
        }
    }
    bool ok = true;
    const int o1 = (ty + 1) * KB1 + tx + 1;        // own cell in a +-1 tile
    const int o3 = (ty + 3) * KB3 + tx + GM::H3;   // own cell in the q tile
    const real dt = (real)A.scal[S_DT];
    const real alpha = (real)A.alpha;

    int issued = i0 + 1;   // last plane issued
    for (int i = i0; i <= i1; ++i) {
        // planes i-1, i (waited before) and i+1 resident; one block-wide
        // verdict, so that every thread leaves the ring together
        bool w = true;
        if (i == i0) w = xt_wait(&bar[slot_of(i - 1)], parity_of(i - 1)) && xt_wait(&bar[slot_of(i)], parity_of(i));
        w = w && xt_wait(&bar[slot_of(i + 1)], parity_of(i + 1));
        if (!__syncthreads_and(w)) {
            ok = false;
            break;
        }
        // every thread is past plane i-2 (read last in the previous step):
        // its slot takes plane i+2, the last plane this block needs being i1+1
        if (i + 2 <= i1 + 1) {
            if (tid == 0) issue(i + 2);
            issued = i + 2;
        }
        // the next plane's x-window values
        real qn = 0, xan = 0, xbn = 0, pgv = 0, hmv = 0;
        if (live) {
            const long id = (long)i * sx + col;
            if (i + 4 < G.NX) qn = q[id + 4 * sx];
            if (VAR == VU) {
                xan = xa[id + sx];
                xbn = A.cn[id + sx];
            } else if (i + 2 < G.NX) {
                xan = xa[id + 2 * sx];
            }
            if (VAR != VC) pgv = A.pg[id];
            hmv = A.Hm[id];
        }
        if (live) {
            const long id = (long)i * sx + col;
            const real* Q = tile3(i);
            auto T = [&](int a, int dp, int dj, int dk) -> real {
                return tile1(i + dp, a)[o1 + dj * KB1 + dk];
            };
            auto QT = [&](int dj, int dk) -> real { return Q[o3 + dj * KB3 + dk]; };
            const real hf = (real)0.5, qr = (real)0.25;
            // advecting velocities (adv_vel)
            real ux, uy, uz;
            if (VAR == VC) {
                ux = hf * (xa1 + xa0);
                uy = hf * (T(0, 0, 1, 0) + T(0, 0, 0, 0));
                uz = hf * (T(1, 0, 0, 1) + T(1, 0, 0, 0));
            } else if (VAR == VU) {
                ux = qx[3];
                uy = qr * (T(0, -1, 0, 0) + T(0, 0, 0, 0) + T(0, 0, 1, 0) + T(0, -1, 1, 0));
                uz = qr * (T(1, -1, 0, 0) + T(1, 0, 0, 0) + T(1, 0, 0, 1) + T(1, -1, 0, 1));
            } else if (VAR == VV) {
                ux = qr * (T(0, 0, -1, 0) + T(0, 1, -1, 0) + T(0, 0, 0, 0) + T(0, 1, 0, 0));
                uy = qx[3];
                uz = qr * (T(1, 0, -1, 0) + T(1, 0, -1, 1) + T(1, 0, 0, 0) + T(1, 0, 0, 1));
            } else {
                ux = qr * (T(0, 0, 0, -1) + T(0, 1, 0, -1) + T(0, 0, 0, 0) + T(0, 1, 0, 0));
                uy = qr * (T(1, 0, 0, -1) + T(1, 0, 0, 0) + T(1, 0, 1, -1) + T(1, 0, 1, 0));
                uz = qx[3];
            }
            // one stencil window at a time (y, then z) keeps register use low
            const real cx = ux * xt_upwind<0, real>(qx, q, G, R, K, i, ux);
            real cy, cz, qym, qyp, qzm, qzp;
            {
                real vy[7];
#pragma unroll
                for (int t = 0; t < 7; ++t) vy[t] = QT(t - 3, 0);
                cy = uy * xt_upwind<1, real>(vy, q, G, R, K, j, uy);
                qym = vy[2];
                qyp = vy[4];
            }
            {
                real vz[7];
#pragma unroll
                for (int t = 0; t < 7; ++t) vz[t] = QT(0, t - 3);
                cz = uz * xt_upwind<2, real>(vz, q, G, R, K, k, uz);
                qzm = vz[2];
                qzp = vz[4];
            }
            const real ct = cz + cx + cy;
            real H;
            if (VAR == VC) {
                H = -(ct);
            } else {
                real s1, s2, s3, s4;
                if (VAR == VU) {   // tiles: 0 v, 1 w, 2 mu_xy, 3 mu_xz
                    s1 = (real)K.xuv * T(2, 0, 1, 0) * (T(0, 0, 1, 0) - T(0, -1, 1, 0));
                    s2 = (real)K.xuv * T(2, 0, 0, 0) * (T(0, 0, 0, 0) - T(0, -1, 0, 0));
                    s3 = (real)K.xuw * T(3, 0, 0, 1) * (T(1, 0, 0, 1) - T(1, -1, 0, 1));
                    s4 = (real)K.xuw * T(3, 0, 0, 0) * (T(1, 0, 0, 0) - T(1, -1, 0, 0));
                } else if (VAR == VV) {   // tiles: 0 u, 1 w, 2 mu_yz, 3 mu_cell, 4 c
                    s1 = (real)K.xvu * xa1 * (T(0, 1, 0, 0) - T(0, 1, -1, 0));
                    s2 = (real)K.xvu * xa0 * (T(0, 0, 0, 0) - T(0, 0, -1, 0));
                    s3 = (real)K.xvw * T(2, 0, 0, 1) * (T(1, 0, 0, 1) - T(1, 0, -1, 1));
                    s4 = (real)K.xvw * T(2, 0, 0, 0) * (T(1, 0, 0, 0) - T(1, 0, -1, 0));
                } else {   // tiles: 0 u, 1 v, 2 mu_yz, 3 mu_cell
                    s1 = (real)K.xwu * xa1 * (T(0, 1, 0, 0) - T(0, 1, 0, -1));
                    s2 = (real)K.xwu * xa0 * (T(0, 0, 0, 0) - T(0, 0, 0, -1));
                    s3 = (real)K.xwv * T(2, 0, 1, 0) * (T(1, 0, 1, 0) - T(1, 0, 1, -1));
                    s4 = (real)K.xwv * T(2, 0, 0, 0) * (T(1, 0, 0, 0) - T(1, 0, 0, -1));
                }
                H = -ct + s1 - s2 + s3 - s4;
            }
            A.H[id] = H;

            // dt*(gamma H + rho H_old + alpha A q_old + alpha body) (acoef)
            const real conv = rk_comb<real>((real)A.g, H, (real)A.r, hmv);
            real a, c;
            if (VAR == VC) {
                a = c = (real)K.cdx;
            } else if (VAR == VU) {
                a = over_h<real>((real)K.d2x * xa0, K.hx, K.ihx, K.pow2);
                c = over_h<real>((real)K.d2x * xa1, K.hx, K.ihx, K.pow2);
            } else {
                a = over_h<real>((real)K.d1x * xa0, K.hx, K.ihx, K.pow2);
                c = over_h<real>((real)K.d1x * xa1, K.hx, K.ihx, K.pow2);
            }
            real b = -(a + c);
            const real ax = a * qx[2] + b * qx[3] + c * qx[4];
            if (VAR == VC) {
                a = c = (real)K.cdy;
            } else if (VAR == VU) {
                a = over_h<real>((real)K.d1y * T(2, 0, 0, 0), K.hy, K.ihy, K.pow2);
                c = over_h<real>((real)K.d1y * T(2, 0, 1, 0), K.hy, K.ihy, K.pow2);
            } else if (VAR == VV) {
                a = over_h<real>((real)K.d2y * T(3, 0, -1, 0), K.hy, K.ihy, K.pow2);
                c = over_h<real>((real)K.d2y * T(3, 0, 0, 0), K.hy, K.ihy, K.pow2);
            } else {
                a = over_h<real>((real)K.d1y * T(2, 0, 0, 0), K.hy, K.ihy, K.pow2);
                c = over_h<real>((real)K.d1y * T(2, 0, 1, 0), K.hy, K.ihy, K.pow2);
            }
            b = -(a + c);
            const real ay = a * qym + b * qx[3] + c * qyp;
            if (VAR == VC) {
                a = c = (real)K.cdz;
            } else if (VAR == VU) {
                a = over_h<real>((real)K.d1z * T(3, 0, 0, 0), K.hz, K.ihz, K.pow2);
                c = over_h<real>((real)K.d1z * T(3, 0, 0, 1), K.hz, K.ihz, K.pow2);
            } else if (VAR == VV) {
                a = over_h<real>((real)K.d1z * T(2, 0, 0, 0), K.hz, K.ihz, K.pow2);
                c = over_h<real>((real)K.d1z * T(2, 0, 0, 1), K.hz, K.ihz, K.pow2);
            } else {
                a = over_h<real>((real)K.d2z * T(3, 0, 0, -1), K.hz, K.ihz, K.pow2);
                c = over_h<real>((real)K.d2z * T(3, 0, 0, 0), K.hz, K.ihz, K.pow2);
            }
            b = -(a + c);
            const real az = a * qzm + b * qx[3] + c * qzp;
            const real diff = alpha * (ax + ay + az);
            real S;
            if (VAR == VC) {
                S = dt * (conv + diff);
            } else {
                real bf;
                if (VAR == VU) {
                    const real cval = (real)0.5 * (xb1 + xb0);
                    bf = alpha * ((real)K.FxRe * cval - over_h<real>(pgv, K.Re, 1.0 / K.Re, 0));
                } else if (VAR == VV) {
                    const real cval = (real)0.5 * (T(4, 0, 0, 0) + T(4, 0, -1, 0));
                    bf = alpha * ((real)K.FyRe * cval - over_h<real>(pgv, K.Re, 1.0 / K.Re, 0));
                } else {
                    bf = alpha * (-over_h<real>(pgv, K.Re, 1.0 / K.Re, 0));
                }
                S = dt * (conv + diff + bf);
            }
            A.S[id] = S;
        }
        // slide the windows one plane along x
#pragma unroll
        for (int t = 0; t < 6; ++t) qx[t] = qx[t + 1];
        qx[6] = qn;
        xa0 = xa1;
        xa1 = xan;
        if (VAR == VU) {
            xb0 = xb1;
            xb1 = xbn;
        }
    }
    if (!ok && tid == 0) {
        // a wait ran out: report it, and drain (bounded) every copy this
        // block issued before its shared memory goes away
        atomicOr(status, ST_TIMEOUT);
        for (int p = i0 - 1; p <= issued; ++p) (void)xt_wait(&bar[slot_of(p)], parity_of(p));
    }
}

}  // namespace
}  // namespace pll
