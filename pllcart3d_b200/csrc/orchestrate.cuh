// Orchestration of the step (pllcart3d.c:156-196), templated on the storage
// type: stage launchers, the substep/step sequences, start-up and the
// per-routine entry points.  form_f64.cu (compiled without multiply-add
// contraction) and form_f32.cu (with) each instantiate one precision form
// and export it through the functions declared in forms.h.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <type_traits>

#include "explicit_tma.cuh"
#include "fft_dct.cuh"
#include "forms.h"
#include "host_common.cuh"
#include "umma_dct.cuh"

namespace pll {
namespace {

// RK3 (Wray) coefficients, global_variables.h:17-18
const double kRK1[3] = {(8.0 / 15.0), (5.0 / 12.0), (3.0 / 4.0)};
const double kRK2[3] = {(0.0), (-17.0 / 60.0), (-5.0 / 12.0)};

// ---- stage launchers --------------------------------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled();

// 3-d tensor map of one padded field ([i][j][k], k contiguous, row pitch sy,
// plane pitch sx) with boxes of box_k x box_j x 1 elements; zeros outside
template <typename real>
bool field_map(CUtensorMap* m, const real* base, const Geo& G, int box_k, int box_j)
{
    EncodeTiledFn fn = encode_tiled();
    if (!fn || ((uintptr_t)base & 15) || (G.sy * (long)sizeof(real)) % 16 || (box_k * (int)sizeof(real)) % 16)
        return false;
    const cuuint64_t dims[3] = {(cuuint64_t)G.NZ, (cuuint64_t)G.NY, (cuuint64_t)G.NX};
    const cuuint64_t strides[2] = {(cuuint64_t)(G.sy * (long)sizeof(real)), (cuuint64_t)(G.sx * (long)sizeof(real))};
    const cuuint32_t box[3] = {(cuuint32_t)box_k, (cuuint32_t)box_j, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, sizeof(real) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)base,
              dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the TMA-staged plane-marching explicit operator (explicit_tma.cuh); false
// when a tensor map cannot be made (the caller then runs k_explicit)
template <typename real, int VAR>
bool launch_explicit_tma(pllgpu_ctx* ctx, const ExplicitArgs<real>& A)
{
    using GM = XtGeom<real>;
    const Rng& R = ctx->Rv[VAR];
    XtMaps M;
    std::memset(&M, 0, sizeof(M));
    const real* staged[5] = {};
    if (VAR == VC) {
        staged[0] = A.vn; staged[1] = A.wn;
    } else if (VAR == VU) {
        staged[0] = A.vn; staged[1] = A.wn; staged[2] = A.mu.xy; staged[3] = A.mu.xz;
    } else if (VAR == VV) {
        staged[0] = A.un; staged[1] = A.wn; staged[2] = A.mu.yz; staged[3] = A.mu.cell; staged[4] = A.cn;
    } else {
        staged[0] = A.un; staged[1] = A.vn; staged[2] = A.mu.yz; staged[3] = A.mu.cell;
    }
    if (!field_map<real>(&M.q, A.q, ctx->G, GM::KB3, GM::JB3)) return false;
    for (int a = 0; a < XtSet<VAR>::NA; ++a)
        if (!field_map<real>(&M.a[a], staged[a], ctx->G, GM::KB1, GM::JB1)) return false;
    const dim3 grid((ctx->G.nz + XT_TK - 1) / XT_TK, (nj(R) + XT_TJ - 1) / XT_TJ, (ni(R) + XT_NI - 1) / XT_NI);
    go<NoBatch>(ctx, k_explicit_tma<VAR, real>, grid, XT_THREADS, XtSmem<real, VAR>::DYN, M, ctx->G, R, ctx->K, A,
                                                                                     ctx->status);
    return true;
}

template <typename real, int VAR>
void launch_explicit(pllgpu_ctx* ctx, const real* un, const real* vn, const real* wn, double g, double r)
{
    static const char* lab[4] = {"explicit_c", "explicit_u", "explicit_v", "explicit_w"};
    const Rng& R = ctx->Rv[VAR];
    ExplicitArgs<real> A;
    A.q = q_old<real>(ctx, VAR);
    A.un = un;
    A.vn = vn;
    A.wn = wn;
    A.mu = mu_old<real>(ctx);
    A.cn = q_new<real>(ctx, VC);
    A.pg = VAR == VC ? nullptr : bufs<real>(ctx).pg[VAR];
    A.Hm = h_nm1<real>(ctx, VAR);
    A.H = h_n<real>(ctx, VAR);
    A.S = bufs<real>(ctx).S;
    A.scal = ctx->scal;
    A.g = g;
    A.r = r;
    A.alpha = g + r;
    int bx, by;
    tune_exp_block(ctx->tune_exp, bx, by);
    if constexpr (std::is_same<real, float>::value) {
        if (ctx->P.explicit_kernel == 2 && !ctx->P.exact_dct && launch_explicit_tma<real, VAR>(ctx, A)) {
            mark(ctx, lab[VAR]);
            return;
        }
        // cell pairs (k, k + EP_DK): blocks of EP_DK x rows, the same threads
        // per block as the tuned shape
        const dim3 blk(EP_DK, bx * by / EP_DK);
        const dim3 grid((nk(R) + 2 * EP_DK - 1) / (2 * EP_DK), (nj(R) + blk.y - 1) / blk.y, ni(R));
        go<k_explicit2_b<VAR>>(ctx, k_explicit2<VAR>, grid, blk, 0, ctx->G, R, ctx->K, A);
    } else {
        if (!ctx->xt_on || ctx->P.explicit_kernel == 1 || !launch_explicit_tma<real, VAR>(ctx, A)) {
            const dim3 blk(bx, by);
            go<k_explicit_b<VAR, real>>(ctx, k_explicit<VAR, real>, box_grid(nk(R), nj(R), ni(R), blk), blk, 0, ctx->G,
                                        R, ctx->K, A);
        }
    }
    mark(ctx, lab[VAR]);
}

// the precision form's segmented solve along x (AXIS 0) or y (AXIS 1):
// lines of P * RS rows or one fewer, P = 16 segments of RS rows, RS in
// {4, 8, 16, 32} ({4, 8, 16} for an FP64 instantiation: a thread holds its
// segment's rows in registers); false: not applicable.  (32 segments of
// 16 rows for 512-row lines measured slower in FP32: at 1024 threads a block
// spills its 16-row registers.)
template <int VAR, int AXIS, int P, int RS, typename real>
void line_seg(pllgpu_ctx* ctx, const Rng& R, const XsweepArgs<real>& X, int n)
{
    const dim3 grid((nk(R) + 31) / 32, AXIS == 0 ? nj(R) : ni(R)), blk(32 * P);
    constexpr size_t smem = line_seg_smem<VAR, AXIS, P, RS, real>();
    if (n == P * RS)
        go<k_line_seg_b<VAR, AXIS, P, RS, true, real>>(ctx, k_line_seg<VAR, AXIS, P, RS, true, real>, grid, blk, smem,
                                                       ctx->G, R, ctx->K, X);
    else
        go<k_line_seg_b<VAR, AXIS, P, RS, false, real>>(ctx, k_line_seg<VAR, AXIS, P, RS, false, real>, grid, blk, smem,
                                                        ctx->G, R, ctx->K, X);
}

template <int VAR, int AXIS, typename real>
bool launch_line_seg(pllgpu_ctx* ctx, const Rng& R, const XsweepArgs<real>& X)
{
    if (ctx->P.exact_dct || ctx->nelem >= (1L << 31)) return false;
    const int n = AXIS == 0 ? ni(R) : nj(R);
    constexpr int p = 16;
    const int rs = (n + p - 1) / p;   // rows per segment
    constexpr bool f32 = std::is_same<real, float>::value;
    if (rs != 4 && rs != 8 && rs != 16 && !(f32 && rs == 32)) return false;
    if (n != p * rs) {
        // one row short: the kernel loads the row past the line (and the
        // viscosity family one beyond it), which must lie in the padded box
        const int start = AXIS == 0 ? R.is : R.js, top = AXIS == 0 ? ctx->G.NX - 1 : ctx->G.NY - 1;
        if (n != p * rs - 1 || start + p * rs + LineCoef<VAR, AXIS>::off > top) return false;
    }
    if (rs == 4) line_seg<VAR, AXIS, p, 4, real>(ctx, R, X, n);
    else if (rs == 8) line_seg<VAR, AXIS, p, 8, real>(ctx, R, X, n);
    else if (rs == 16) line_seg<VAR, AXIS, p, 16, real>(ctx, R, X, n);
    else if constexpr (f32) line_seg<VAR, AXIS, p, 32, real>(ctx, R, X, n);
    return true;
}

// shared-memory opt-in of the segmented solves (static separator arrays and
// dynamic row tiles together pass the 48 KB default: FP32 from 16 rows per
// segment, FP64 from 4)
template <int VAR, int AXIS, int P, int RS, typename real>
void line_seg_attr()
{
    const int b = (int)line_seg_smem<VAR, AXIS, P, RS, real>();
    cudaFuncSetAttribute(k_line_seg<VAR, AXIS, P, RS, true, real>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    cudaFuncSetAttribute(k_line_seg<VAR, AXIS, P, RS, false, real>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}

template <int VAR, typename real>
void line_seg_attrs()
{
    line_seg_attr<VAR, 0, 16, 4, real>();
    line_seg_attr<VAR, 1, 16, 4, real>();
    line_seg_attr<VAR, 0, 16, 8, real>();
    line_seg_attr<VAR, 0, 16, 16, real>();
    line_seg_attr<VAR, 1, 16, 8, real>();
    line_seg_attr<VAR, 1, 16, 16, real>();
    if constexpr (std::is_same<real, float>::value) {
        line_seg_attr<VAR, 0, 16, 32, real>();
        line_seg_attr<VAR, 1, 16, 32, real>();
    }
}

template <typename real, int VAR>
void launch_implicit(pllgpu_ctx* ctx, double g, double r)
{
    static const char* ly[4] = {"adi_y_c", "adi_y_u", "adi_y_v", "adi_y_w"};
    static const char* lz[4] = {"adi_z_c", "adi_z_u", "adi_z_v", "adi_z_w"};
    static const char* lx[4] = {"adi_x_c", "adi_x_u", "adi_x_v", "adi_x_w"};
    const Rng& R = ctx->Rv[VAR];
    const double alpha = g + r;
    Bufs<real>& B = bufs<real>(ctx);
    XsweepArgs<real> X;
    X.mu = mu_new<real>(ctx);
    X.q = q_old<real>(ctx, VAR);
    X.qn = q_new<real>(ctx, VAR);
    X.H = h_n<real>(ctx, VAR);
    X.Hm = h_nm1<real>(ctx, VAR);
    X.S = B.S;
    X.cc = B.cc;
    X.scal = ctx->scal;
    X.g = g;
    X.r = r;
    X.alpha = alpha;
    const int lb = tune_line_block(ctx->tune_line);
    bool ydone = false;
    if constexpr (!std::is_same<real, float>::value && !PLL_FP64_EXACT && VAR == VC) {
        // FP64 forms: the segmented y solve for concentration (0.65 against
        // 0.95 ms per step at 512x256x256).  For momentum, whose segments
        // also stage viscosity rows, one 512-thread block per SM measured
        // slower than the prefetching sweep (1.12 against 1.00 ms).
        ydone = launch_line_seg<VAR, 1, real>(ctx, R, X);
    }
    if constexpr (std::is_same<real, float>::value) {
        // the precision form's partitioned solves: segmented when the line
        // length allows, else for concentration the warp solve of short
        // lines
        ydone = launch_line_seg<VAR, 1, real>(ctx, R, X);
        if (!ydone && VAR == VC && nj(R) <= ZP_MAX && nj(R) >= 2 * (ZP_MAX / 32) && !ctx->P.exact_dct) {
            go<k_adi_y_part_b<VAR, float>>(ctx, k_adi_y_part<VAR, float>, dim3((nk(R) + 31) / 32, ni(R)), 256,
                                           adi_y_part_smem<float>(), ctx->G, R, ctx->K, X.mu, B.S, ctx->scal, alpha);
            ydone = true;
        }
    }
    if (!ydone)
        go<k_line_pf_b<VAR, 1, real>>(ctx, k_line_pf<VAR, 1, real>, dim3((nk(R) + lb - 1) / lb, ni(R)), lb, 0, ctx->G,
                                      R, ctx->K, X);
    mark(ctx, ly[VAR]);
    bool zdone = false;
    if constexpr (std::is_same<real, float>::value || !PLL_FP64_EXACT) {
        if (nk(R) <= ZP_MAX && nk(R) >= 2 * (ZP_MAX / 32) && !ctx->P.exact_dct) {
            // the partitioned warp solve (precision form and FP64 form)
            go<k_adi_z_part_b<VAR, real>>(ctx, k_adi_z_part<VAR, real>, dim3((nj(R) + 3) / 4, ni(R)), 128, 0, ctx->G, R,
                                          ctx->K, X.mu, B.S, ctx->scal, alpha);
            zdone = true;
        }
    }
    if (!zdone) {
        constexpr size_t smem = adi_z_smem_bytes<VAR, real>();
        go<k_adi_z_tiled_b<VAR, real>>(ctx, k_adi_z_tiled<VAR, real>, dim3((nj(R) + 127) / 128, ni(R)), 128, smem,
                                       ctx->G, R, ctx->K, X.mu, B.S, B.cc, ctx->scal, alpha);
    }
    mark(ctx, lz[VAR]);
    bool xdone = false;
    if constexpr (std::is_same<real, float>::value) xdone = launch_line_seg<VAR, 0, real>(ctx, R, X);
    if (!xdone)
        go<k_line_pf_b<VAR, 0, real>>(ctx, k_line_pf<VAR, 0, real>, dim3((nk(R) + lb - 1) / lb, nj(R)), lb, 0, ctx->G,
                                      R, ctx->K, X);
    mark(ctx, lx[VAR]);
}

template <typename real>
void launch_viscosity(pllgpu_ctx* ctx, const real* cn, MuPtrs<real> m, int law = -1)
{
    dim3 blk(32, 4);
    if constexpr (std::is_same<real, float>::value || !PLL_FP64_EXACT) {
        if ((law < 0 ? ctx->P.nmvp : law) == 0) {   // the exponential law on cell pairs
            const dim3 grid((ctx->G.NZ + 2 * EP_DK - 1) / (2 * EP_DK), (ctx->G.NY + blk.y - 1) / blk.y,
                            (ni(ctx->Rg) + 2 + VISC_NI - 1) / VISC_NI);
            go<k_viscosity2_b<real>>(ctx, k_viscosity2<real>, grid, blk, 0, ctx->G, ctx->Rg, ctx->K, cn, (real*)m.cell,
                                     (real*)m.xy, (real*)m.xz, (real*)m.yz);
            mark(ctx, "viscosity");
            return;
        }
    }
    go<k_viscosity_b<real>>(ctx, k_viscosity<real>,
                            box_grid(ctx->G.NZ, ctx->G.NY, (ni(ctx->Rg) + 2 + VISC_NI - 1) / VISC_NI, blk), blk, 0,
                            ctx->G, ctx->Rg, ctx->K, law < 0 ? ctx->P.nmvp : law, cn, (real*)m.cell, (real*)m.xy,
                            (real*)m.xz, (real*)m.yz, ctx->scal);
    mark(ctx, "viscosity");
}

void launch_gemm(pllgpu_ctx* ctx, const GemmDesc& d, const double* A, const double* B, double* C)
{
    dim3 grid((d.N + 63) / 64, (d.M + 63) / 64, d.batch);
    if (ctx->P.exact_dct)
        go<k_gemm_seq_b<double>>(ctx, k_gemm_seq<double>, grid, 256, 0, d, A, B, C);
    else
        go<k_gemm_dmma_b>(ctx, k_gemm_dmma, grid, 256, 0, d, A, B, C);
    mark(ctx, "dct_gemm");
}

void launch_gemm(pllgpu_ctx* ctx, const GemmDesc& d, const float* A, const float* B, float* C)
{
    dim3 grid((d.N + 63) / 64, (d.M + 63) / 64, d.batch);
    if (ctx->P.exact_dct)
        go<k_gemm_seq_b<float>>(ctx, k_gemm_seq<float>, grid, 256, 0, d, A, B, C);
    else
        go<k_gemm_tf32x3_b>(ctx, k_gemm_tf32x3, grid, 256, 0, d, A, B, C);
    mark(ctx, "dct_gemm");
}

// one tcgen05 DCT pass over all planes (pass 0 forward z, 1 forward y,
// 2 inverse y, 3 inverse z); rows = planes x rows per plane, K = the
// transform length = the output columns
void launch_umma(pllgpu_ctx* ctx, int pass, long rows, int K, const UmmaEpi& e, float* out)
{
    const UmmaPlan& U = ctx->um;
    const int ntiles = (int)(rows / UM_BM);
    if (e.rows_per_plane % UM_BM) {   // the epilogue assumes whole tiles per plane
        fail(ctx, PLLGPU_EINVAL);
        return;
    }
    if (ctx->P.dct_kernel == 2) {   // one tile per CTA
        const dim3 grid((unsigned)ntiles);
        if (K == 256)
            go<NoBatch>(ctx, k_dct_umma<256>, grid, UM_THREADS, UmmaSmem<256>::DYN, U.a[pass], U.bh[pass], U.bl[pass],
                                                                               K, e, out, ctx->status);
        else
            go<NoBatch>(ctx, k_dct_umma<128>, grid, UM_THREADS, UmmaSmem<128>::DYN, U.a[pass], U.bh[pass], U.bl[pass],
                                                                               K, e, out, ctx->status);
    } else {   // persistent: one CTA per SM
        const dim3 grid((unsigned)std::min(ntiles, U.sms));
        if (K == 256)
            go<NoBatch>(ctx, k_dct_umma_p<256>, grid, UMP_THREADS, UmmaPSmem<256>::DYN, U.a[pass], U.bh[pass],
                        U.bl[pass], K, ntiles, e, out, ctx->status);
        else
            go<NoBatch>(ctx, k_dct_umma_p<128>, grid, UMP_THREADS, UmmaPSmem<128>::DYN, U.a[pass], U.bh[pass],
                        U.bl[pass], K, ntiles, e, out, ctx->status);
    }
    mark(ctx, "dct_umma");
}

void launch_poisson_umma(pllgpu_ctx* ctx)
{
    Bufs<float>& B = ctx->b32;
    const int nx = ctx->G.nx, ny = ctx->G.ny, nz = ctx->G.nz;
    const long N = (long)ny * nz;
    // forward z: dct2[x][kz][y] = sum_z dct1[x][y][z] Tz[kz][z] (stored transposed)
    launch_umma(ctx, 0, (long)nx * ny, nz, UmmaEpi{ny, N, 1, ny, 1.f, 0, 1}, B.dct2);
    // forward y: dct1[x][kz][ky] = sum_y dct2[x][kz][y] Ty[ky][y]
    launch_umma(ctx, 1, (long)nx * nz, ny, UmmaEpi{nz, N, ny, 1, 1.f, 0, 0}, B.dct1);
    go<k_poisson_x2_b>(ctx, k_poisson_x2, (int)((N + 127) / 128), 128, 0, nx, ny, nz, ctx->K, ctx->lam_y, ctx->lam_z,
                       B.dct1, (float*)ctx->mode_rr, ctx->mode_cc, 1);
    mark(ctx, "poisson_x");
    // inverse y: dct2[x][y][kz] = sum_ky dct1[x][kz][ky] Tiy[y][ky] (stored transposed)
    launch_umma(ctx, 2, (long)nx * nz, ny, UmmaEpi{nz, N, 1, nz, 1.f, 0, 1}, B.dct2);
    // inverse z into phi's interior, divided by 4*ny*nz
    const double four_n = (double)(4 * N);
    const bool p2 = is_pow2(four_n);
    float* phi0 = B.phi + (long)ctx->Rg.is * ctx->G.sx + (long)ctx->Rg.js * ctx->G.sy + ctx->Rg.ks;
    launch_umma(ctx, 3, (long)nx * ny, nz,
                UmmaEpi{ny, ctx->G.sx, ctx->G.sy, 1, (float)(p2 ? 1.0 / four_n : four_n), p2 ? 1 : 2, 0}, phi0);
}

#if !PLL_FP64_EXACT
// lengths the FFT passes take: powers of two with whole 16-line tiles
inline bool fft_len_ok(int n) { return n >= 16 && n <= 256 && (n & (n - 1)) == 0; }

template <int N, int KIND, bool CONTIG>
void fft_launch(pllgpu_ctx* ctx, const FftLines& d, int axis, const double* in, double* out)
{
    const unsigned grid = (unsigned)(d.lines / (2 * FFT_PB));
    go<k_dct_fft_b<double, N, KIND, CONTIG>>(ctx, k_dct_fft<double, N, KIND, CONTIG>, grid, FFT_THREADS,
                                             fft_smem_bytes<N>(), d, in, out, ctx->fft_tw[axis], ctx->fft_wq[axis]);
}

template <int KIND, bool CONTIG>
void fft_pass(pllgpu_ctx* ctx, int N, const FftLines& d, int axis, const double* in, double* out)
{
    switch (N) {
    case 16: fft_launch<16, KIND, CONTIG>(ctx, d, axis, in, out); break;
    case 32: fft_launch<32, KIND, CONTIG>(ctx, d, axis, in, out); break;
    case 64: fft_launch<64, KIND, CONTIG>(ctx, d, axis, in, out); break;
    case 128: fft_launch<128, KIND, CONTIG>(ctx, d, axis, in, out); break;
    default: fft_launch<256, KIND, CONTIG>(ctx, d, axis, in, out); break;
    }
    mark(ctx, "dct_fft");
}

// the FP64 form's Poisson solve with FFT DCT passes (compact [x][y][z])
void launch_poisson_fft(pllgpu_ctx* ctx)
{
    Bufs<double>& B = ctx->b64;
    const int nx = ctx->G.nx, ny = ctx->G.ny, nz = ctx->G.nz;
    const long N = (long)ny * nz;
    // y lines: (x, z) -> x*N + z, elements step nz; z lines: (x, y) -> x*N + y*nz
    const FftLines ylines{nx * nz, nz, N, 1, nz, N, 1, nz, 1.0};
    const FftLines zlines{nx * ny, ny, N, nz, 1, N, nz, 1, 1.0};
    fft_pass<0, false>(ctx, ny, ylines, 0, B.dct1, B.dct2);
    fft_pass<0, true>(ctx, nz, zlines, 1, B.dct2, B.dct1);
    go<k_poisson_x_b<double>>(ctx, k_poisson_x<double>, (int)((N + 127) / 128), 128, 0, nx, ny, nz, ctx->K,
                              ctx->lam_y, ctx->lam_z, B.dct1, ctx->mode_cc, ctx->mode_rr, 0);
    mark(ctx, "poisson_x");
    fft_pass<1, false>(ctx, ny, ylines, 0, B.dct1, B.dct2);
    // into phi's interior, times 1/(4 ny nz) (exact: a power of two)
    FftLines out = zlines;
    out.sa_out = ctx->G.sx;
    out.sb_out = ctx->G.sy;
    out.scale = 1.0 / (4.0 * (double)N);
    double* phi0 = B.phi + (long)ctx->Rg.is * ctx->G.sx + (long)ctx->Rg.js * ctx->G.sy + ctx->Rg.ks;
    fft_pass<1, true>(ctx, nz, out, 1, B.dct2, phi0);
}
#endif

// phisolver_dct after its right-hand side is in dct1 (compact [x][y][z])
template <typename real>
void launch_poisson(pllgpu_ctx* ctx)
{
    if constexpr (std::is_same<real, float>::value) {
        if (ctx->um.on) {
            launch_poisson_umma(ctx);
            return;
        }
    } else {
#if !PLL_FP64_EXACT
        if (ctx->fft_on) {
            launch_poisson_fft(ctx);
            return;
        }
#endif
    }
    Bufs<real>& B = bufs<real>(ctx);
    const int nx = ctx->G.nx, ny = ctx->G.ny, nz = ctx->G.nz;
    const long N = (long)ny * nz;
    GemmDesc d{};
    // forward, y pass: dct2[x][ky][z] = sum_y Ty[ky][y] dct1[x][y][z]
    d = GemmDesc{ny, nz, ny, nx, 0, ny, 1, N, nz, 1, N, nz, 1, 0.0, 0};
    launch_gemm(ctx, d, B.Ty, B.dct1, B.dct2);
    // forward, z pass: dct1[x][ky][kz] = sum_z dct2[x][ky][z] Tz[kz][z]
    d = GemmDesc{ny, nz, nz, nx, N, nz, 1, 0, 1, nz, N, nz, 1, 0.0, 0};
    launch_gemm(ctx, d, B.dct2, B.Tz, B.dct1);
    // x-tridiagonal per mode, in place in dct1, FP64 arithmetic
    go<k_poisson_x_b<real>>(ctx, k_poisson_x<real>, (int)((N + 127) / 128), 128, 0, nx, ny, nz, ctx->K,
                            ctx->lam_y, ctx->lam_z, B.dct1, ctx->mode_cc, ctx->mode_rr, 0);
    mark(ctx, "poisson_x");
    // inverse, y pass: dct2[x][y][kz] = sum_ky Tiy[y][ky] dct1[x][ky][kz]
    d = GemmDesc{ny, nz, ny, nx, 0, ny, 1, N, nz, 1, N, nz, 1, 0.0, 0};
    launch_gemm(ctx, d, B.Tiy, B.dct1, B.dct2);
    // inverse, z pass into phi's interior, divided by 4*ny*nz
    const double four_n = (double)(4 * N);
    d = GemmDesc{ny, nz, nz, nx, N, nz, 1, 0, 1, nz, ctx->G.sx, ctx->G.sy, 1,
                 is_pow2(four_n) ? 1.0 / four_n : four_n, is_pow2(four_n) ? 1 : 2};
    real* phi0 = B.phi + (long)ctx->Rg.is * ctx->G.sx + (long)ctx->Rg.js * ctx->G.sy + ctx->Rg.ks;
    launch_gemm(ctx, d, B.dct2, B.Tiz, phi0);
}

template <typename real>
void launch_phi_ghosts(pllgpu_ctx* ctx)
{
    const Rng& R = ctx->Rg;
    real* phi = bufs<real>(ctx).phi;
    go<k_phi_ghosts_b<0, real>>(ctx, k_phi_ghosts<0, real>, dim3((nj(R) + 127) / 128, ni(R)), 128, 0, ctx->G, R, phi);
    mark(ctx, "phi_ghosts");
    go<k_phi_ghosts_b<1, real>>(ctx, k_phi_ghosts<1, real>, dim3((nk(R) + 127) / 128, ni(R)), 128, 0, ctx->G, R, phi);
    mark(ctx, "phi_ghosts");
    go<k_phi_ghosts_b<2, real>>(ctx, k_phi_ghosts<2, real>, dim3((nk(R) + 127) / 128, nj(R)), 128, 0, ctx->G, R, phi);
    mark(ctx, "phi_ghosts");
}

template <typename real>
void launch_project(pllgpu_ctx* ctx, double alpha, int correct, int ghosts, int pgu)
{
    Bufs<real>& B = bufs<real>(ctx);
    const MuPtrs<real> mu = mu_new<real>(ctx);
    dim3 blk(32, 4);
    if constexpr (std::is_same<real, float>::value || !PLL_FP64_EXACT) {
        const dim3 grid((nk(ctx->Rg) + 2 * EP_DK - 1) / (2 * EP_DK), (nj(ctx->Rg) + blk.y - 1) / blk.y,
                        ni(ctx->Rg) + 1);
        go<k_project2_b<real>>(ctx, k_project2<real>, grid, blk, 0, ctx->G, ctx->Rg, ctx->Rv[VU], ctx->Rv[VV],
                               ctx->Rv[VW], ctx->K, q_new<real>(ctx, VU), q_new<real>(ctx, VV), q_new<real>(ctx, VW),
                               B.pg[VU], B.pg[VV], B.pg[VW], B.phi, mu, ctx->scal, alpha, correct, ghosts, pgu);
        mark(ctx, "project");
        return;
    }
    go<k_project_b<real>>(ctx, k_project<real>,
                          box_grid(nk(ctx->Rg), nj(ctx->Rg), (ni(ctx->Rg) + 1 + PROJECT_NI - 1) / PROJECT_NI, blk), blk,
                          0, ctx->G, ctx->Rg, ctx->Rv[VU], ctx->Rv[VV], ctx->Rv[VW], ctx->K, q_new<real>(ctx, VU),
                          q_new<real>(ctx, VV), q_new<real>(ctx, VW), B.pg[VU], B.pg[VV], B.pg[VW], B.phi, mu.cell,
                          mu.xy, mu.xz, mu.yz, ctx->scal, alpha, correct, ghosts, pgu);
    mark(ctx, "project");
}

template <typename real>
void launch_div(pllgpu_ctx* ctx, int mode, double alpha)
{
    Bufs<real>& B = bufs<real>(ctx);
    dim3 blk(32, 4);
    if constexpr (std::is_same<real, float>::value || !PLL_FP64_EXACT) {
        if (mode == 0) {   // the right-hand side on cell pairs
            const dim3 grid((nk(ctx->Rg) + 2 * EP_DK - 1) / (2 * EP_DK), (nj(ctx->Rg) + blk.y - 1) / blk.y,
                            (ni(ctx->Rg) + DIV_NI - 1) / DIV_NI);
            go<k_div_rhs2_b<real>>(ctx, k_div_rhs2<real>, grid, blk, 0, ctx->G, ctx->Rg, ctx->K, q_new<real>(ctx, VU),
                                   q_new<real>(ctx, VV), q_new<real>(ctx, VW), B.dct1, ctx->scal, alpha);
            mark(ctx, "div_rhs");
            return;
        }
    }
    go<k_div_rhs_b<real>>(ctx, k_div_rhs<real>, box_grid(nk(ctx->Rg), nj(ctx->Rg), ni(ctx->Rg), blk), blk, 0, ctx->G,
                          ctx->Rg, ctx->K, q_new<real>(ctx, VU), q_new<real>(ctx, VV), q_new<real>(ctx, VW), B.div,
                          B.div, B.dct1, ctx->scal, alpha, mode);
    mark(ctx, "div_rhs");
}

template <typename real>
void launch_flux(pllgpu_ctx* ctx)
{
    if constexpr (std::is_same<real, float>::value) {
        const int rows = 2 * nj(ctx->Rv[VU]);
        go<k_flux3_b>(ctx, k_flux3, (rows + 31) / 32, 1024, 0, ctx->G, ctx->Rv[VU], ctx->K, q_new<real>(ctx, VU),
                      ctx->red, ctx->ticket, ctx->scal);
        mark(ctx, "flux");
        return;
    }
    go<k_flux_b<real>>(ctx, k_flux<real>, 1, 512, sizeof(double) * 2 * ctx->G.NY, ctx->G, ctx->Rv[VU], ctx->K,
                                                                       q_new<real>(ctx, VU), ctx->scal);
    mark(ctx, "flux");
}

template <typename real>
void launch_bulk(pllgpu_ctx* ctx)
{
    go<k_bulk2_b<real>>(ctx, k_bulk2<real>, BULK_BLOCKS, 1024, 0, ctx->G, ctx->Rg, q_old<real>(ctx, VU), ctx->red,
                                                      ctx->ticket + 1, ctx->scal);
    mark(ctx, "bulk_velo");
}

template <typename real>
void launch_cfl(pllgpu_ctx* ctx)
{
    dim3 blk(32, 8);
    if constexpr (std::is_same<real, float>::value) {
        const dim3 grid((nk(ctx->Rg) + 2 * EP_DK - 1) / (2 * EP_DK), (nj(ctx->Rg) + blk.y - 1) / blk.y,
                        (ni(ctx->Rg) + CFL_NI - 1) / CFL_NI);
        go<k_cfl2_b>(ctx, k_cfl2, grid, blk, 0, ctx->G, ctx->Rg, ctx->K, q_old<real>(ctx, VU), q_old<real>(ctx, VV),
                                          q_old<real>(ctx, VW), ctx->scal, ctx->status);
    } else {
        go<k_cfl_b<real>>(ctx, k_cfl<real>, box_grid(nk(ctx->Rg), nj(ctx->Rg), ni(ctx->Rg), blk), blk, 0, ctx->G,
                          ctx->Rg, ctx->K, q_old<real>(ctx, VU), q_old<real>(ctx, VV), q_old<real>(ctx, VW), ctx->scal,
                          ctx->status);
    }
    mark(ctx, "cfl");
    go<k_dt_b>(ctx, k_dt, 1, 1, 0, ctx->K, ctx->scal);
    mark(ctx, "dt");
}

// one RK3-CN substep of the fast path, pllcart3d.c:164-194
template <typename real>
void enqueue_substep(pllgpu_ctx* ctx, int rk)
{
    const double g = kRK1[rk], r = kRK2[rk], alpha = g + r;
    const real *uo = q_old<real>(ctx, VU), *vo = q_old<real>(ctx, VV), *wo = q_old<real>(ctx, VW);
    launch_bulk<real>(ctx);
    // concentration: advected by u->new == u->old
    launch_explicit<real, VC>(ctx, uo, vo, wo, g, r);
    launch_implicit<real, VC>(ctx, g, r);
    launch_viscosity<real>(ctx, q_new<real>(ctx, VC), mu_new<real>(ctx));
    launch_explicit<real, VU>(ctx, uo, vo, wo, g, r);
    launch_implicit<real, VU>(ctx, g, r);
    launch_explicit<real, VV>(ctx, uo, vo, wo, g, r);
    launch_implicit<real, VV>(ctx, g, r);
    launch_explicit<real, VW>(ctx, uo, vo, wo, g, r);
    launch_implicit<real, VW>(ctx, g, r);
    // update_velo_boundary (L182) writes only ghost entries that nothing
    // reads before update_veloghost_points (L189) rewrites them; skipped
    launch_flux<real>(ctx);
    launch_div<real>(ctx, 0, alpha);
    launch_poisson<real>(ctx);
    launch_phi_ghosts<real>(ctx);
    launch_project<real>(ctx, alpha, 1, 1, 1);
    ctx->cur ^= 1;  // update_old_*: roles swap
    if (ctx->resync_c) {
        // After a restart the reference's c->new holds values its routines
        // never write (intermediate() restores c->old only, pllcart3d.c:3209)
        // and update_old_conc copies them into c->old after this substep;
        // one full copy makes the two buffers agree there from now on.
        if (cudaMemcpyAsync(q_new<real>(ctx, VC), q_old<real>(ctx, VC), sizeof(real) * (size_t)ctx->nelem,
                            cudaMemcpyDeviceToDevice, ctx->st) != cudaSuccess)
            fail(ctx, PLLGPU_ECUDA);
        ctx->resync_c = false;
    }
}

__device__ __forceinline__ void k_tval_run(const uint3, const dim3, double* scal, double a0, double a1, double a2)
{
    // tval += (gamma+rho) dt per substep, pllcart3d.c:166
    const double dt = scal[S_DT];
    double t = scal[S_TVAL];
    t = t + a0 * dt;
    t = t + a1 * dt;
    t = t + a2 * dt;
    scal[S_TVAL] = t;
}
__global__ void k_tval(double* scal, double a0, double a1, double a2)
{
    k_tval_run(blockIdx, gridDim, scal, a0, a1, a2);
}
struct k_tval_b {
    static constexpr auto run = &k_tval_run;
    static constexpr int maxt = 0, minb = 0;
};

template <typename real>
void enqueue_step(pllgpu_ctx* ctx)
{
    launch_cfl<real>(ctx);
    for (int rk = 0; rk < 3; ++rk) enqueue_substep<real>(ctx, rk);
    go<k_tval_b>(ctx, k_tval, 1, 1, 0, ctx->scal, kRK1[0] + kRK2[0], kRK1[1] + kRK2[1], kRK1[2] + kRK2[2]);
    mark(ctx, "tval");
}

template <typename real>
int materialize_t(pllgpu_ctx* ctx)
{
    const size_t bytes = sizeof(real) * (size_t)ctx->nelem;
    Bufs<real>& B = bufs<real>(ctx);
    for (int v = 0; v < 4; ++v) {
        CK(cudaMemcpyAsync(q_new<real>(ctx, v), q_old<real>(ctx, v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(h_n<real>(ctx, v), h_nm1<real>(ctx, v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(B.mu[1 - ctx->cur][v], B.mu[ctx->cur][v], bytes, cudaMemcpyDeviceToDevice, ctx->st));
    }
    return PLLGPU_OK;
}

template <typename real>
real* field_ptr_raw(pllgpu_ctx* ctx, int f)
{
    if (f < 0 || f >= PLLGPU_NFIELDS) return nullptr;
    Bufs<real>& B = bufs<real>(ctx);
    if (f <= PLLGPU_C_HNM1) {
        const int r = f - PLLGPU_C_OLD;
        return r == 0 ? q_old<real>(ctx, VC) : r == 1 ? q_new<real>(ctx, VC) : r == 2 ? h_n<real>(ctx, VC)
                                                                             : h_nm1<real>(ctx, VC);
    }
    if (f <= PLLGPU_W_PG) {
        const int v = 1 + (f - PLLGPU_U_OLD) / 5, r = (f - PLLGPU_U_OLD) % 5;
        return r == 0 ? q_old<real>(ctx, v) : r == 1 ? q_new<real>(ctx, v) : r == 2 ? h_n<real>(ctx, v)
             : r == 3 ? h_nm1<real>(ctx, v) : B.pg[v];
    }
    if (f <= PLLGPU_MU_OLD_YZ) return B.mu[ctx->cur][f - PLLGPU_MU_OLD_CELL];
    if (f <= PLLGPU_MU_NEW_YZ) return B.mu[1 - ctx->cur][f - PLLGPU_MU_NEW_CELL];
    if (f == PLLGPU_PHI) return B.phi;
    return B.div;
}

// ---- start-up, routines ---------------------------------------------------------

// start-up of pllcart3d.c:75-142.  fresh: after an initial condition
// (ghosts, then new -> old); otherwise after intermediate() restored the
// state (L111), where only the viscosity start-up follows.
template <typename real>
int start_t(pllgpu_ctx* ctx, bool fresh = true)
{
    const size_t bytes = sizeof(real) * (size_t)ctx->nelem;
    if (fresh) {
        // update_ghost_points (L81) on the initial velocities; phi is zero
        launch_project<real>(ctx, 0.0, 0, 1, 0);
        // update_old_conc / update_old_velo (L82-83): both buffers equal
        for (int v = 0; v < 4; ++v) {
            CK(cudaMemcpyAsync(q_old<real>(ctx, v), q_new<real>(ctx, v), bytes, cudaMemcpyDeviceToDevice,
                               ctx->st));
            CK(cudaMemcpyAsync(h_nm1<real>(ctx, v), h_n<real>(ctx, v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
        }
    }
    if (ctx->P.nmvp) {
        const double PI = 4.0 * std::atan(1.0);
        // slope_parameter reads FP64 c (pllcart3d.c:133); the mixed form
        // widens its FP32 c through the staging field
        const double* c64 = nullptr;
        if (ctx->mixed) {
            k_convert_to_f64<<<(int)((ctx->nelem + 255) / 256), 256, 0, ctx->st>>>(
                ctx->nelem, (const float*)q_new<real>(ctx, VC), ctx->stage64);
            c64 = ctx->stage64;
        } else {
            c64 = (const double*)q_new<real>(ctx, VC);
        }
        k_slope_parameter<<<1, 1, 0, ctx->st>>>(ctx->G, ctx->Rg, ctx->P.Y1, ctx->P.Z1, ctx->G.dy, ctx->G.dz,
                                                ctx->P.Vratio, ctx->P.Mum, ctx->P.Lambda, PI, c64, ctx->scal,
                                                ctx->status, ctx->work);
    }
    // calculate_viscosity(c->old, mu_old), L142
    launch_viscosity<real>(ctx, q_old<real>(ctx, VC), mu_old<real>(ctx));
    return PLLGPU_OK;
}

int set_dt_vb(pllgpu_ctx* ctx, double dt, double vb)
{
    if (set_scalar(ctx, S_DT, dt) || set_scalar(ctx, S_VBULK, vb)) return ctx->err;
    return PLLGPU_OK;
}

template <typename real>
int routine_t(pllgpu_ctx* ctx, int routine, const double* in, double* out)
{
    const double dt = in ? in[0] : 0.0, g = in ? in[1] : 0.0, r = in ? in[2] : 0.0, vb = in ? in[3] : 0.0;
    const double alpha = g + r;
    const size_t bytes = sizeof(real) * (size_t)ctx->nelem;
    Bufs<real>& B = bufs<real>(ctx);
    switch (routine) {
    case PLLGPU_R_CONCENTRATION:
        if (set_dt_vb(ctx, dt, vb)) return ctx->err;
        launch_explicit<real, VC>(ctx, q_new<real>(ctx, VU), q_new<real>(ctx, VV), q_new<real>(ctx, VW), g, r);
        launch_implicit<real, VC>(ctx, g, r);
        break;
    case PLLGPU_R_VISCOSITY_NEW:
        launch_viscosity<real>(ctx, q_new<real>(ctx, VC), mu_new<real>(ctx));
        break;
    case PLLGPU_R_XMOM:
    case PLLGPU_R_YMOM:
    case PLLGPU_R_ZMOM: {
        if (set_dt_vb(ctx, dt, vb)) return ctx->err;
        const real *uo = q_old<real>(ctx, VU), *vo = q_old<real>(ctx, VV), *wo = q_old<real>(ctx, VW);
        if (routine == PLLGPU_R_XMOM) {
            launch_explicit<real, VU>(ctx, uo, vo, wo, g, r);
            launch_implicit<real, VU>(ctx, g, r);
        } else if (routine == PLLGPU_R_YMOM) {
            launch_explicit<real, VV>(ctx, uo, vo, wo, g, r);
            launch_implicit<real, VV>(ctx, g, r);
        } else {
            launch_explicit<real, VW>(ctx, uo, vo, wo, g, r);
            launch_implicit<real, VW>(ctx, g, r);
        }
        break;
    }
    case PLLGPU_R_VELO_GHOSTS:
        launch_project<real>(ctx, 0.0, 0, 1, 0);
        break;
    case PLLGPU_R_DIVERGENCE:
        launch_div<real>(ctx, 1, 0.0);
        break;
    case PLLGPU_R_PHISOLVER:
        if (set_scalar(ctx, S_DT, dt)) return ctx->err;
        launch_div<real>(ctx, 2, alpha);
        launch_poisson<real>(ctx);
        break;
    case PLLGPU_R_PHI_GHOSTS:
        launch_phi_ghosts<real>(ctx);
        break;
    case PLLGPU_R_VELO_CORRECTION:
        if (set_scalar(ctx, S_DT, dt)) return ctx->err;
        launch_flux<real>(ctx);
        launch_project<real>(ctx, alpha, 1, 0, 0);
        break;
    case PLLGPU_R_PRESSURE_GRADIENT:
        if (set_scalar(ctx, S_DT, dt)) return ctx->err;
        launch_project<real>(ctx, alpha, 0, 0, 1);
        break;
    case PLLGPU_R_ROTATE:
        for (int v = 0; v < 4; ++v) {
            CK(cudaMemcpyAsync(q_old<real>(ctx, v), q_new<real>(ctx, v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
            CK(cudaMemcpyAsync(h_nm1<real>(ctx, v), h_n<real>(ctx, v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
            CK(cudaMemcpyAsync(B.mu[ctx->cur][v], B.mu[1 - ctx->cur][v], bytes, cudaMemcpyDeviceToDevice, ctx->st));
        }
        break;
    case PLLGPU_R_BULK_VELO:
        launch_bulk<real>(ctx);
        if (out) out[0] = get_scalar(ctx, S_VBULK);
        break;
    case PLLGPU_R_FIND_CFL:
        // find_cfl's own return value CFLmax/max (before the Timestep clip)
        launch_cfl<real>(ctx);
        if (out) out[0] = get_scalar(ctx, S_CFLDT);
        break;
    case PLLGPU_R_SUBSTEP: {
        const int rk = (int)g;
        if (rk < 0 || rk > 2) return fail(ctx, PLLGPU_EINVAL);
        if (set_scalar(ctx, S_DT, dt)) return ctx->err;
        enqueue_substep<real>(ctx, rk);
        ctx->rotated = true;
        break;
    }
    case PLLGPU_R_VISCOSITY_EXP:
        launch_viscosity<real>(ctx, q_new<real>(ctx, VC), mu_new<real>(ctx), 0);
        break;
    case PLLGPU_R_VISCOSITY_NMVP: {
        // coefficients of calculate_viscosity_nmvp (pllcart3d.c:895-900)
        const double cm = dt, PI = 4.0 * std::atan(1.0), M = ctx->P.Vratio;
        const double alp = std::exp(M), mum = ctx->P.Mum * alp;
        const double psi0 = std::asin(alp / mum), psi1 = PI - std::asin(1 / mum);
        const double etam = (PI / 2 - psi0) / (psi1 - psi0);
        const double a = ((1 - cm) - etam) / ((1 - cm) * (etam - 1));
        if (set_scalar(ctx, S_CM, cm) || set_scalar(ctx, S_MUM, mum) || set_scalar(ctx, S_PSI0, psi0) ||
            set_scalar(ctx, S_PSI1, psi1) || set_scalar(ctx, S_NMVA, a))
            return ctx->err;
        launch_viscosity<real>(ctx, q_new<real>(ctx, VC), mu_new<real>(ctx), 1);
        break;
    }
    case PLLGPU_R_SLOPE_PARAMETER: {
        if (ctx->mixed) return fail(ctx, PLLGPU_EINVAL);
        const double PI = 4.0 * std::atan(1.0);
        k_slope_parameter<<<1, 1, 0, ctx->st>>>(ctx->G, ctx->Rg, ctx->P.Y1, ctx->P.Z1, ctx->G.dy, ctx->G.dz,
                                                ctx->P.Vratio, ctx->P.Mum, ctx->P.Lambda, PI,
                                                (const double*)q_new<real>(ctx, VC), ctx->scal, ctx->status,
                                                ctx->work);
        mark(ctx, "slope_parameter");
        if (out) out[0] = get_scalar(ctx, S_CM);
        break;
    }
    default:
        return fail(ctx, PLLGPU_EINVAL);
    }
    return PLLGPU_OK;
}

// FP64 diagnostics: mass, divergence norms, mixing length
__global__ void k_diag_final(int nplanes, int ny, int nz, double dV, double dx, const double* __restrict__ pl,
                             double* __restrict__ out)
{
    double mass = 0.0, dmax = 0.0, d2 = 0.0, lmix = 0.0;
    for (int i = 0; i < nplanes; ++i) {
        const double sc = pl[3 * i], cbar = sc / ((double)ny * (double)nz);
        mass += sc * dV;
        dmax = fmax(dmax, pl[3 * i + 1]);
        d2 += pl[3 * i + 2];
        if (cbar > 0.01 && cbar < 0.99) lmix += dx;
    }
    out[0] = mass;
    out[1] = dmax;
    out[2] = sqrt(d2 * dV);
    out[3] = lmix;
}

template <typename real>
void launch_diag(pllgpu_ctx* ctx)
{
    const Rng& R = ctx->Rg;
    k_plane_diag<real><<<ni(R), 256, 0, ctx->st>>>(ctx->G, R, ctx->K, q_old<real>(ctx, VC), q_old<real>(ctx, VU),
                                                   q_old<real>(ctx, VV), q_old<real>(ctx, VW), ctx->diag);
    const double dV = ctx->G.dx * ctx->G.dy * ctx->G.dz;
    k_diag_final<<<1, 1, 0, ctx->st>>>(ni(R), ctx->G.ny, ctx->G.nz, dV, ctx->G.dx, ctx->diag,
                                       ctx->diag + 3L * ni(R));
}

// ---- tcgen05 DCT set-up (precision form) ----------------------------------------

// TF32 round-to-nearest, ties away from zero, of a finite float
float tf32_rna_host(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u = (u + 0x1000u) & ~0x1FFFu;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}


EncodeTiledFn encode_tiled()
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

// row-major FP32 matrix [rows][cols], boxes of 32 columns x box_rows rows,
// 128-byte swizzle (the shared-memory layout tcgen05 reads as K-major SW128)
bool tile_map(CUtensorMap* m, const float* base, long rows, int cols, int box_rows)
{
    EncodeTiledFn fn = encode_tiled();
    if (!fn || ((uintptr_t)base & 15) || (cols * 4) % 16 || cols % UM_BK || box_rows > 256) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 4};
    const cuuint32_t box[2] = {(cuuint32_t)UM_BK, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)base, dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool setup_umma(pllgpu_ctx* c)
{
    Bufs<float>& B = c->b32;
    UmmaPlan& U = c->um;
    const int nx = c->P.nx, ny = c->P.ny, nz = c->P.nz;
    // pass: A buffer, A rows, transform length, cosine matrix (FP32, [n][k])
    const float* A[4] = {B.dct1, B.dct2, B.dct1, B.dct2};
    const long rows[4] = {(long)nx * ny, (long)nx * nz, (long)nx * nz, (long)nx * ny};
    const int len[4] = {nz, ny, ny, nz};
    const float* T[4] = {B.Tz, B.Ty, B.Tiy, B.Tiz};
    for (int p = 0; p < 4; ++p) {
        const long n2 = (long)len[p] * len[p];
        std::vector<float> t((size_t)n2), hi((size_t)n2), lo((size_t)n2);
        if (cudaMemcpy(t.data(), T[p], sizeof(float) * n2, cudaMemcpyDeviceToHost) != cudaSuccess) return false;
        for (long i = 0; i < n2; ++i) {
            hi[i] = tf32_rna_host(t[i]);
            lo[i] = tf32_rna_host(t[i] - hi[i]);
        }
        if (!(U.Thi[p] = dalloc<float>(c, n2)) || !(U.Tlo[p] = dalloc<float>(c, n2))) return false;
        cudaMemcpy(U.Thi[p], hi.data(), sizeof(float) * n2, cudaMemcpyHostToDevice);
        cudaMemcpy(U.Tlo[p], lo.data(), sizeof(float) * n2, cudaMemcpyHostToDevice);
        if (!tile_map(&U.a[p], A[p], rows[p], len[p], UM_BM) || !tile_map(&U.bh[p], U.Thi[p], len[p], len[p], len[p]) ||
            !tile_map(&U.bl[p], U.Tlo[p], len[p], len[p], len[p]))
            return false;
    }
    if (cudaFuncSetAttribute(k_dct_umma<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)UmmaSmem<256>::DYN) != cudaSuccess ||
        cudaFuncSetAttribute(k_dct_umma<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)UmmaSmem<128>::DYN) != cudaSuccess ||
        cudaFuncSetAttribute(k_dct_umma_p<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)UmmaPSmem<256>::DYN) != cudaSuccess ||
        cudaFuncSetAttribute(k_dct_umma_p<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)UmmaPSmem<128>::DYN) != cudaSuccess ||
        cudaDeviceGetAttribute(&U.sms, cudaDevAttrMultiProcessorCount, c->dev) != cudaSuccess)
        return false;
    U.on = true;
    return true;
}

#if !PLL_FP64_EXACT
// twiddle tables of the FFT DCT passes, evaluated in long double and
// rounded once (arguments reduced exactly: m < N, k < N)
bool setup_fft(pllgpu_ctx* c)
{
    const int len[2] = {c->P.ny, c->P.nz};
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int a = 0; a < 2; ++a) {
        const int N = len[a];
        std::vector<double2> tw((size_t)N), wq((size_t)N);
        for (int m = 0; m < N; ++m) {
            const long double t = 2.0L * pi * (long double)m / (long double)N;
            tw[m] = make_double2((double)cosl(t), (double)sinl(t));
            const long double q = pi * (long double)m / (2.0L * (long double)N);
            wq[m] = make_double2((double)cosl(q), (double)sinl(q));
        }
        c->fft_tw[a] = (double2*)dalloc<double>(c, 2L * N);
        c->fft_wq[a] = (double2*)dalloc<double>(c, 2L * N);
        if (!c->fft_tw[a] || !c->fft_wq[a]) return false;
        if (cudaMemcpy(c->fft_tw[a], tw.data(), sizeof(double2) * N, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(c->fft_wq[a], wq.data(), sizeof(double2) * N, cudaMemcpyHostToDevice) != cudaSuccess)
            return false;
    }
    c->fft_on = true;
    return true;
}
#endif

template <typename real>
bool alloc_state(pllgpu_ctx* c)
{
    Bufs<real>& B = bufs<real>(c);
    const pllgpu_params* p = &c->P;
    bool ok = true;
    for (int v = 0; v < 4 && ok; ++v)
        for (int b = 0; b < 2 && ok; ++b)
            ok = (B.q[v][b] = dalloc<real>(c, c->nelem)) && (B.H[v][b] = dalloc<real>(c, c->nelem));
    for (int b = 0; b < 2 && ok; ++b)
        for (int m = 0; m < 4 && ok; ++m) ok = (B.mu[b][m] = dalloc<real>(c, c->nelem)) != nullptr;
    for (int v = 1; v < 4 && ok; ++v) ok = (B.pg[v] = dalloc<real>(c, c->nelem)) != nullptr;
    const long ncell = (long)p->nx * p->ny * p->nz;
    ok = ok && (B.phi = dalloc<real>(c, c->nelem)) && (B.div = dalloc<real>(c, c->nelem)) &&
         (B.S = dalloc<real>(c, c->nelem)) && (B.cc = dalloc<real>(c, c->nelem)) &&
         (B.dct1 = dalloc<real>(c, ncell)) && (B.dct2 = dalloc<real>(c, ncell)) &&
         (B.Ty = dalloc<real>(c, (long)p->ny * p->ny)) && (B.Tz = dalloc<real>(c, (long)p->nz * p->nz)) &&
         (B.Tiy = dalloc<real>(c, (long)p->ny * p->ny)) && (B.Tiz = dalloc<real>(c, (long)p->nz * p->nz));
    if (!ok) return false;
    std::vector<real> T((size_t)std::max(p->ny, p->nz) * std::max(p->ny, p->nz));
    dct_matrix<real>(0, p->ny, T.data());
    cudaMemcpy(B.Ty, T.data(), sizeof(real) * p->ny * p->ny, cudaMemcpyHostToDevice);
    dct_matrix<real>(0, p->nz, T.data());
    cudaMemcpy(B.Tz, T.data(), sizeof(real) * p->nz * p->nz, cudaMemcpyHostToDevice);
    dct_matrix<real>(1, p->ny, T.data());
    cudaMemcpy(B.Tiy, T.data(), sizeof(real) * p->ny * p->ny, cudaMemcpyHostToDevice);
    dct_matrix<real>(1, p->nz, T.data());
    cudaMemcpy(B.Tiz, T.data(), sizeof(real) * p->nz * p->nz, cudaMemcpyHostToDevice);
    // kernels above the 48 KB default of dynamic shared memory
    if constexpr (std::is_same<real, float>::value) {
        cudaFuncSetAttribute(k_adi_y_part<VC, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)adi_y_part_smem<float>());
        cudaFuncSetAttribute(k_adi_y_part<VU, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)adi_y_part_smem<float>());
        cudaFuncSetAttribute(k_adi_y_part<VV, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)adi_y_part_smem<float>());
        cudaFuncSetAttribute(k_adi_y_part<VW, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)adi_y_part_smem<float>());
    }
    if constexpr (!std::is_same<real, float>::value && !PLL_FP64_EXACT) line_seg_attrs<VC, real>();
    if constexpr (std::is_same<real, float>::value) {
        line_seg_attrs<VC, real>();
        line_seg_attrs<VU, real>();
        line_seg_attrs<VV, real>();
        line_seg_attrs<VW, real>();
    }
    cudaFuncSetAttribute(k_adi_z_tiled<VC, real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)adi_z_smem_bytes<VC, real>());
    cudaFuncSetAttribute(k_adi_z_tiled<VU, real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)adi_z_smem_bytes<VU, real>());
    cudaFuncSetAttribute(k_adi_z_tiled<VV, real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)adi_z_smem_bytes<VV, real>());
    cudaFuncSetAttribute(k_adi_z_tiled<VW, real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)adi_z_smem_bytes<VW, real>());
    if constexpr (std::is_same<real, float>::value) {
        if (p->explicit_kernel == 2) {
            cudaFuncSetAttribute(k_explicit_tma<VC, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 XtSmem<float, VC>::DYN);
            cudaFuncSetAttribute(k_explicit_tma<VU, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 XtSmem<float, VU>::DYN);
            cudaFuncSetAttribute(k_explicit_tma<VV, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 XtSmem<float, VV>::DYN);
            cudaFuncSetAttribute(k_explicit_tma<VW, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 XtSmem<float, VW>::DYN);
        }
        const bool shape_ok = (p->ny == 128 || p->ny == 256) && (p->nz == 128 || p->nz == 256);
        if (shape_ok && !p->exact_dct && p->dct_kernel != 1 && !setup_umma(c)) return false;
    } else {
#if !PLL_FP64_EXACT
        if (!p->exact_dct && fft_len_ok(p->ny) && fft_len_ok(p->nz) && !setup_fft(c)) return false;
        if (!p->exact_dct && c->nelem < (1L << 31) && encode_tiled()) {
            cudaFuncSetAttribute(k_explicit_tma<VC, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 XtSmem<double, VC>::DYN);
            cudaFuncSetAttribute(k_explicit_tma<VU, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 XtSmem<double, VU>::DYN);
            cudaFuncSetAttribute(k_explicit_tma<VV, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 XtSmem<double, VV>::DYN);
            cudaFuncSetAttribute(k_explicit_tma<VW, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 XtSmem<double, VW>::DYN);
            c->xt_on = true;
        }
#endif
    }
    return true;
}

}  // namespace
}  // namespace pll

// exported entry points of one precision form
#define PLL_DEFINE_FORM(SUFFIX, REAL)                                                          \
    namespace pll {                                                                          \
    void form_enqueue_step_##SUFFIX(pllgpu_ctx* c) { enqueue_step<REAL>(c); }                \
    int form_start_##SUFFIX(pllgpu_ctx* c) { return start_t<REAL>(c); }                      \
    int form_resume_##SUFFIX(pllgpu_ctx* c) { return start_t<REAL>(c, false); }              \
    int form_routine_##SUFFIX(pllgpu_ctx* c, int r, const double* in, double* out)           \
    {                                                                                        \
        return routine_t<REAL>(c, r, in, out);                                               \
    }                                                                                        \
    int form_materialize_##SUFFIX(pllgpu_ctx* c) { return materialize_t<REAL>(c); }          \
    void* form_field_ptr_##SUFFIX(pllgpu_ctx* c, int f) { return (void*)field_ptr_raw<REAL>(c, f); } \
    void form_diag_##SUFFIX(pllgpu_ctx* c) { launch_diag<REAL>(c); }                         \
    bool form_alloc_##SUFFIX(pllgpu_ctx* c) { return alloc_state<REAL>(c); }                 \
    }
