// Device context, step orchestration and the pllgpu_ C ABI.
//
// The reference advances its state with one routine call per stage
// (pllcart3d.c:158-195) and copies new -> old after every RK substep
// (update_old_*, L3402-3452).  Here the state lives in HBM for the whole
// run, each stage is one or a few kernels on one stream, the new/old,
// H^n/H^{n-1} and mu_new/mu_old pairs are ping-pong buffers whose roles swap
// instead of being copied, and a whole time step is replayed as one CUDA
// graph (two graphs, one per buffer parity).
//
// Swapping is equivalent to the reference's copies because (a) every entry
// of a "new" array that a substep writes is written every substep, (b) the
// entries it never writes (IC ghosts, wall faces, the inlet face) are equal
// in both buffers from pllgpu_start on, and (c) the one read of "new"
// before it is written in a substep - the advecting velocities of
// concentration (pllcart3d.c:171 passes u->new, which equals u->old then) -
// reads the "old" buffer instead.  The per-routine entry points keep the
// reference's copy semantics exactly (PLLGPU_R_ROTATE copies).
//
// Two forms share the orchestration, templated on the storage type:
// PLLGPU_FP64 keeps every field in FP64 (the reference's arithmetic);
// PLLGPU_MIXED keeps the state in FP32 (WENO fluxes, stress terms, ADI
// sweeps in FP32), runs the DCT passes as split-TF32 tensor-core GEMMs with
// FP32 accumulation, and keeps FP64 for the Poisson mode solve (eigenvalue
// division, zero mode and gauge) and for the CFL, flux, mass and divergence
// reductions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/pllcart3d_gpu.h"
#include "forms.h"
#include "host_common.cuh"

using namespace pll;

// one entry point of the context's form: the precision form (FP32 state),
// the exact FP64 form (exact_dct), the FP64 form with FP32 WENO weights, or
// the FP64 form
#define FORM_CALL(c, fn, ...)                                                                          \
    ((c)->mixed                                 ? fn##_f32(__VA_ARGS__)                              \
     : (c)->P.exact_dct                         ? fn##_f64x(__VA_ARGS__)                             \
     : (c)->P.precision == PLLGPU_MIXED64       ? fn##_f64m(__VA_ARGS__)                             \
                                                : fn##_f64(__VA_ARGS__))

namespace pll {

void enqueue_step_any(pllgpu_ctx* ctx) { FORM_CALL(ctx, form_enqueue_step, ctx); }

namespace {

int build_graphs(pllgpu_ctx* ctx)
{
    for (int t = 0; t < 2; ++t) {
        const int c0 = ctx->cur;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
        ctx->counting = 0;
        enqueue_step_any(ctx);
        CK(cudaStreamEndCapture(ctx->st, &g));
        ctx->launches_per_step = ctx->counting;
        CK(cudaGraphInstantiate(&ctx->gexec[c0], g, 0));
        cudaGraphDestroy(g);
        // cur flipped once by the three substeps
    }
    ctx->graphs_ready = true;
    return PLLGPU_OK;
}

// ---- field access -------------------------------------------------------------

// After fast steps the reference's state has new == old (update_old_*
// copies); the ping-pong buffers hold a stale "new".  Reads of new-role
// fields then see the old-role buffer; writes first copy old -> new.
bool is_new_role(int f)
{
    return f == PLLGPU_C_NEW || f == PLLGPU_C_HN || f == PLLGPU_U_NEW || f == PLLGPU_U_HN ||
           f == PLLGPU_V_NEW || f == PLLGPU_V_HN || f == PLLGPU_W_NEW || f == PLLGPU_W_HN ||
           (f >= PLLGPU_MU_NEW_CELL && f <= PLLGPU_MU_NEW_YZ);
}

int new_to_old(int f)
{
    switch (f) {
    case PLLGPU_C_NEW: return PLLGPU_C_OLD;
    case PLLGPU_C_HN: return PLLGPU_C_HNM1;
    case PLLGPU_U_NEW: return PLLGPU_U_OLD;
    case PLLGPU_U_HN: return PLLGPU_U_HNM1;
    case PLLGPU_V_NEW: return PLLGPU_V_OLD;
    case PLLGPU_V_HN: return PLLGPU_V_HNM1;
    case PLLGPU_W_NEW: return PLLGPU_W_OLD;
    case PLLGPU_W_HN: return PLLGPU_W_HNM1;
    default: return f - (PLLGPU_MU_NEW_CELL - PLLGPU_MU_OLD_CELL);
    }
}

template <int VAR>
__global__ void k_acoef(Geo G, Rng R, Consts K, MuPtrs<double> mu, double* __restrict__ abc, long nelem)
{
    const int k = R.ks + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = R.js + blockIdx.y * blockDim.y + threadIdx.y;
    const int i = R.is + blockIdx.z;
    if (k > R.ke || j > R.je) return;
    const long id = (long)i * G.sx + (long)j * G.sy + k;
    double a, b, c;
    acoef<VAR, 0, double>(K, G, mu.cell, mu.xy, mu.xz, mu.yz, id, a, b, c);
    abc[id] = a; abc[nelem + id] = b; abc[2 * nelem + id] = c;
    acoef<VAR, 1, double>(K, G, mu.cell, mu.xy, mu.xz, mu.yz, id, a, b, c);
    abc[3 * nelem + id] = a; abc[4 * nelem + id] = b; abc[5 * nelem + id] = c;
    acoef<VAR, 2, double>(K, G, mu.cell, mu.xy, mu.xz, mu.yz, id, a, b, c);
    abc[6 * nelem + id] = a; abc[7 * nelem + id] = b; abc[8 * nelem + id] = c;
}


}  // namespace
}  // namespace pll

namespace pll {

static int materialize_t_any(pllgpu_ctx* ctx)
{
    return FORM_CALL(ctx, form_materialize, ctx);
}

int materialize(pllgpu_ctx* ctx)
{
    if (!ctx->rotated) return PLLGPU_OK;
    int e = materialize_t_any(ctx);
    if (e) return e;
    CK(cudaStreamSynchronize(ctx->st));
    ctx->rotated = false;
    return PLLGPU_OK;
}

void* field_ptr(pllgpu_ctx* ctx, int f, bool for_write)
{
    if (f < 0 || f >= PLLGPU_NFIELDS) return nullptr;
    if (ctx->rotated && is_new_role(f)) {
        if (!for_write) f = new_to_old(f);
        else if (materialize(ctx)) return nullptr;
    }
    return FORM_CALL(ctx, form_field_ptr, ctx, f);
}

}  // namespace pll

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* pllgpu_error_string(int code)
{
    switch (code) {
    case PLLGPU_OK: return "ok";
    case PLLGPU_ENAN: return "NaN or Inf in the velocity field";
    case PLLGPU_ECUDA: return "CUDA error";
    case PLLGPU_ETIMEOUT: return "device wait timed out";
    case PLLGPU_EBOUNDS: return "index out of bounds";
    case PLLGPU_EINVAL: return "invalid argument";
    case PLLGPU_ENOCONV: return "slope-parameter bisection did not converge";
    default: return "unknown";
    }
}

pllgpu_ctx* pllgpu_create(const pllgpu_params* p, int device)
{
    if (!p || p->nx < 4 || p->ny < 4 || p->nz < 4) return nullptr;
    if (p->precision != PLLGPU_FP64 && p->precision != PLLGPU_MIXED && p->precision != PLLGPU_MIXED64)
        return nullptr;
    pllgpu_ctx* ctx = new pllgpu_ctx();
    ctx->P = *p;
    ctx->dev = device;
    ctx->mixed = p->precision == PLLGPU_MIXED;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return nullptr;
    }
    Geo& G = ctx->G;
    G.nx = p->nx; G.ny = p->ny; G.nz = p->nz;
    G.NX = p->nx + 6; G.NY = p->ny + 2; G.NZ = p->nz + 2;
    G.sy = ((G.NZ + 7) / 8) * 8;
    G.sx = (long)G.NY * G.sy;
    // grid_setup, pllcart3d.c:380-382
    G.dx = (p->X2 - p->X1) / (double)p->nx;
    G.dy = (p->Y2 - p->Y1) / (double)p->ny;
    G.dz = (p->Z2 - p->Z1) / (double)p->nz;
    ctx->nelem = (long)G.NX * G.sx;
    if (ctx->nelem >= (1L << 31)) {   // kernels index a field with 32-bit offsets
        cudaStreamDestroy(ctx->st);
        delete ctx;
        return nullptr;
    }
    // index ranges, simulation_setup pllcart3d.c:405-431 (one rank)
    Rng& Rg = ctx->Rg;
    Rg.is = 3; Rg.ie = p->nx + 2; Rg.js = 1; Rg.je = p->ny; Rg.ks = 1; Rg.ke = p->nz;
    for (int v = 0; v < 4; ++v) ctx->Rv[v] = Rg;
    ctx->Rv[VU].is = Rg.is + 1;
    ctx->Rv[VV].js = Rg.js + 1;
    ctx->Rv[VW].ks = Rg.ks + 1;
    // constants, each the reference's own expression
    Consts& K = ctx->K;
    const double Re = p->Re, Pe = p->Pe;
    K.hx = G.dx; K.hy = G.dy; K.hz = G.dz;
    K.pow2 = is_pow2(G.dx) && is_pow2(G.dy) && is_pow2(G.dz);
    K.ihx = 1.0 / G.dx; K.ihy = 1.0 / G.dy; K.ihz = 1.0 / G.dz;
    K.i2hx = 1.0 / (2.0 * G.dx); K.i2hy = 1.0 / (2.0 * G.dy); K.i2hz = 1.0 / (2.0 * G.dz);
    K.cdx = 1.0 / (Pe * G.dx * G.dx);
    K.cdy = 1.0 / (Pe * G.dy * G.dy);
    K.cdz = 1.0 / (Pe * G.dz * G.dz);
    K.d1x = 1.0 / (Re * G.dx); K.d1y = 1.0 / (Re * G.dy); K.d1z = 1.0 / (Re * G.dz);
    K.d2x = 2.0 / (Re * G.dx); K.d2y = 2.0 / (Re * G.dy); K.d2z = 2.0 / (Re * G.dz);
    K.xuv = 1.0 / (Re * G.dy * G.dx); K.xuw = 1.0 / (Re * G.dz * G.dx);
    K.xvu = 1.0 / (Re * G.dx * G.dy); K.xvw = 1.0 / (Re * G.dz * G.dy);
    K.xwu = 1.0 / (Re * G.dx * G.dz); K.xwv = 1.0 / (Re * G.dy * G.dz);
    K.FxRe = -(p->Fx / Re);
    K.FyRe = -(p->Fy / Re);
    K.Re = Re;
    K.area = (p->Y2 - p->Y1) * (p->Z2 - p->Z1);
    K.dx2i = 1.0 / (G.dx * G.dx);
    K.CFLmax = p->CFLmax;
    K.M = p->Vratio;
    K.Vnorm = 0.0;

    pllgpu_ctx* c = ctx;
    const long ncell = (long)p->nx * p->ny * p->nz;
    bool ok = FORM_CALL(ctx, form_alloc, c);
    ok = ok && (c->mode_cc = dalloc<double>(c, ncell)) && (c->mode_rr = dalloc<double>(c, ncell)) &&
         (c->lam_y = dalloc<double>(c, p->ny)) && (c->lam_z = dalloc<double>(c, p->nz)) &&
         (c->scal = dalloc<double>(c, S_COUNT)) && (c->work = dalloc<double>(c, 2L * (p->nx + 8))) &&
         (c->diag = dalloc<double>(c, 3L * p->nx + 8)) && (c->status = dalloc<int>(c, 1)) &&
         (c->red = dalloc<double>(c, red_doubles(c->G))) && (c->ticket = dalloc<unsigned>(c, 2));
    if (ok && ctx->mixed) ok = (c->stage64 = dalloc<double>(c, c->nelem)) != nullptr;
    if (!ok) {
        pllgpu_destroy(ctx);
        return nullptr;
    }
    // Poisson eigenvalues (phisolver_dct L2050-2051)
    {
        const double PI = 4.0 * std::atan(1.0);
        std::vector<double> ly(p->ny), lz(p->nz);
        for (int j = 0; j < p->ny; ++j)
            ly[j] = 2.0 * (std::cos(PI * (double)j / (double)p->ny) - 1.0) / (G.dy * G.dy);
        for (int k = 0; k < p->nz; ++k)
            lz[k] = 2.0 * (std::cos(PI * (double)k / (double)p->nz) - 1.0) / (G.dz * G.dz);
        cudaMemcpy(c->lam_y, ly.data(), sizeof(double) * p->ny, cudaMemcpyHostToDevice);
        cudaMemcpy(c->lam_z, lz.data(), sizeof(double) * p->nz, cudaMemcpyHostToDevice);
    }
    // Timestep with the diffusive cap of pllcart3d.c:150-154
    {
        double dmin = (G.dx < G.dy) ? G.dx : G.dy;
        dmin = (dmin < G.dz) ? dmin : G.dz;
        double diff_dt = 0.1 * p->Pe * dmin * dmin;
        c->timestep = (diff_dt < p->Timestep) ? diff_dt : p->Timestep;
        cudaMemcpy(c->scal + S_TIMESTEP, &c->timestep, sizeof(double), cudaMemcpyHostToDevice);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) {
        pllgpu_destroy(ctx);
        return nullptr;
    }
    return ctx;
}

void pllgpu_destroy(pllgpu_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->dev);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    for (int t = 0; t < 2; ++t)
        if (ctx->gexec[t]) cudaGraphExecDestroy(ctx->gexec[t]);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    for (void* p : ctx->allocs) cudaFree(p);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
}

int pllgpu_field_id(const char* name)
{
    static const char* names[PLLGPU_NFIELDS] = {
        "c_old", "c_new", "c_hn", "c_hnm1",
        "u_old", "u_new", "u_hn", "u_hnm1", "u_pg",
        "v_old", "v_new", "v_hn", "v_hnm1", "v_pg",
        "w_old", "w_new", "w_hn", "w_hnm1", "w_pg",
        "mu_old_cell", "mu_old_xy", "mu_old_xz", "mu_old_yz",
        "mu_new_cell", "mu_new_xy", "mu_new_xz", "mu_new_yz",
        "phi", "div"};
    if (!name) return -1;
    for (int i = 0; i < PLLGPU_NFIELDS; ++i)
        if (!std::strcmp(name, names[i])) return i;
    return -1;
}

int pllgpu_dims(const pllgpu_ctx* ctx, int* d)
{
    if (!ctx || !d) return PLLGPU_EINVAL;
    d[0] = ctx->G.NX; d[1] = ctx->G.NY; d[2] = ctx->G.NZ;
    d[3] = ctx->G.nx; d[4] = ctx->G.ny; d[5] = ctx->G.nz;
    return PLLGPU_OK;
}

int pllgpu_set_field(pllgpu_ctx* ctx, int f, const double* host)
{
    if (!ctx || !host) return PLLGPU_EINVAL;
    void* d = field_ptr(ctx, f, true);
    if (!d) return fail(ctx, PLLGPU_EINVAL);
    const Geo& G = ctx->G;
    if (!ctx->mixed) {
        CK(cudaMemcpy2DAsync(d, sizeof(double) * G.sy, host, sizeof(double) * G.NZ, sizeof(double) * G.NZ,
                             (size_t)G.NX * G.NY, cudaMemcpyHostToDevice, ctx->st));
    } else {
        CK(cudaMemcpy2DAsync(ctx->stage64, sizeof(double) * G.sy, host, sizeof(double) * G.NZ,
                             sizeof(double) * G.NZ, (size_t)G.NX * G.NY, cudaMemcpyHostToDevice, ctx->st));
        k_convert_to_f32<<<(int)((ctx->nelem + 255) / 256), 256, 0, ctx->st>>>(ctx->nelem, ctx->stage64, (float*)d);
        if (int e = check_launch(ctx)) return e;
    }
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

int pllgpu_get_field(pllgpu_ctx* ctx, int f, double* host)
{
    if (!ctx || !host) return PLLGPU_EINVAL;
    void* d = field_ptr(ctx, f, false);
    if (!d) return fail(ctx, PLLGPU_EINVAL);
    const Geo& G = ctx->G;
    const double* src = (const double*)d;
    if (ctx->mixed) {
        k_convert_to_f64<<<(int)((ctx->nelem + 255) / 256), 256, 0, ctx->st>>>(ctx->nelem, (const float*)d,
                                                                                ctx->stage64);
        if (int e = check_launch(ctx)) return e;
        src = ctx->stage64;
    }
    CK(cudaMemcpy2DAsync(host, sizeof(double) * G.NZ, src, sizeof(double) * G.sy, sizeof(double) * G.NZ,
                         (size_t)G.NX * G.NY, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

int pllgpu_device_field(pllgpu_ctx* ctx, int f, double** dptr, long* si, long* sj)
{
    if (!ctx) return PLLGPU_EINVAL;
    void* d = field_ptr(ctx, f, true);
    if (!d) return PLLGPU_EINVAL;
    if (dptr) *dptr = (double*)d;
    if (si) *si = ctx->G.sx;
    if (sj) *sj = ctx->G.sy;
    return PLLGPU_OK;
}

int pllgpu_start(pllgpu_ctx* ctx)
{
    if (!ctx) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    if (int e = materialize(ctx)) return e;
    int e = FORM_CALL(ctx, form_start, ctx);
    if (e) return e;
    if (int e2 = check_launch(ctx)) return e2;
    CK(cudaStreamSynchronize(ctx->st));
    set_scalar(ctx, S_TVAL, 0.0);
    return read_status(ctx);
}

int pllgpu_resume(pllgpu_ctx* ctx, double tval)
{
    if (!ctx) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    if (int e = materialize(ctx)) return e;
    int e = FORM_CALL(ctx, form_resume, ctx);
    if (e) return e;
    ctx->resync_c = true;
    if (int e2 = check_launch(ctx)) return e2;
    CK(cudaStreamSynchronize(ctx->st));
    set_scalar(ctx, S_TVAL, tval);
    return read_status(ctx);
}

int pllgpu_steps(pllgpu_ctx* ctx, int nsteps)
{
    if (!ctx || nsteps < 0) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    if (ctx->resync_c && nsteps > 0) {
        // first step after a restart on the stream (it carries one extra copy)
        ctx->counting = 0;
        enqueue_step_any(ctx);
        if (int e = check_launch(ctx)) return e;
        ctx->rotated = true;
        --nsteps;
    }
    if (ctx->P.use_graph) {
        if (!ctx->graphs_ready) {
            if (int e = build_graphs(ctx)) return e;
        }
        for (int s = 0; s < nsteps; ++s) {
            CK(cudaGraphLaunch(ctx->gexec[ctx->cur], ctx->st));
            ctx->cur ^= 1;
        }
    } else {
        for (int s = 0; s < nsteps; ++s) {
            ctx->counting = 0;
            enqueue_step_any(ctx);
            ctx->launches_per_step = ctx->counting;
            if (int e = check_launch(ctx)) return e;
        }
    }
    if (nsteps > 0) ctx->rotated = true;
    CK(cudaStreamSynchronize(ctx->st));
    return read_status(ctx);
}

int pllgpu_autotune(pllgpu_ctx* ctx, int trial_steps, int* steps_done)
{
    if (!ctx || trial_steps < 1) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    if (int e = materialize(ctx)) return e;
    // Every variant computes bit-identical results, so the trials are steps
    // of the run itself: nothing is saved or restored, and the state after
    // tuning equals the state of the same number of untuned steps.
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int best_e = ctx->tune_exp, best_l = ctx->tune_line, done = 0;
    float best = 1e30f;
    if (ctx->resync_c) {   // the restart copy runs on the first step
        enqueue_step_any(ctx);
        ++done;
    }
    for (int ve = 0; ve < NTUNE_EXP; ++ve)
        for (int vl = 0; vl < NTUNE_LINE; ++vl) {
            ctx->tune_exp = ve;
            ctx->tune_line = vl;
            enqueue_step_any(ctx);   // warm-up of this variant
            CK(cudaEventRecord(e0, ctx->st));
            for (int s = 0; s < trial_steps; ++s) enqueue_step_any(ctx);
            CK(cudaEventRecord(e1, ctx->st));
            if (int e = check_launch(ctx)) return e;
            CK(cudaEventSynchronize(e1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            done += trial_steps + 1;
            if (ms < best) {
                best = ms;
                best_e = ve;
                best_l = vl;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->tune_exp = best_e;
    ctx->tune_line = best_l;
    // graphs captured with the old shapes are rebuilt on the next steps call
    for (int t = 0; t < 2; ++t)
        if (ctx->gexec[t]) {
            cudaGraphExecDestroy(ctx->gexec[t]);
            ctx->gexec[t] = nullptr;
        }
    ctx->graphs_ready = false;
    ctx->rotated = true;
    if (steps_done) *steps_done = done;
    CK(cudaStreamSynchronize(ctx->st));
    return read_status(ctx);
}

int pllgpu_tuning(pllgpu_ctx* ctx, int* explicit_variant, int* line_variant)
{
    if (!ctx) return PLLGPU_EINVAL;
    if (explicit_variant) *explicit_variant = ctx->tune_exp;
    if (line_variant) *line_variant = ctx->tune_line;
    return PLLGPU_OK;
}

int pllgpu_set_tuning(pllgpu_ctx* ctx, int explicit_variant, int line_variant)
{
    if (!ctx || explicit_variant < 0 || explicit_variant >= NTUNE_EXP || line_variant < 0 ||
        line_variant >= NTUNE_LINE)
        return PLLGPU_EINVAL;
    ctx->tune_exp = explicit_variant;
    ctx->tune_line = line_variant;
    for (int t = 0; t < 2; ++t)
        if (ctx->gexec[t]) {
            cudaGraphExecDestroy(ctx->gexec[t]);
            ctx->gexec[t] = nullptr;
        }
    ctx->graphs_ready = false;
    return PLLGPU_OK;
}

int pllgpu_copy_state(pllgpu_ctx* dst, pllgpu_ctx* src)
{
    if (!dst || !src || dst == src || dst->mixed != src->mixed || dst->nelem != src->nelem ||
        dst->P.nx != src->P.nx || dst->P.ny != src->P.ny || dst->P.nz != src->P.nz)
        return PLLGPU_EINVAL;
    pllgpu_ctx* ctx = src;   // error reports go to the source context
    CK(cudaSetDevice(src->dev));
    CK(cudaStreamSynchronize(dst->st));
    const size_t esz = src->mixed ? sizeof(float) : sizeof(double);
    const size_t bytes = esz * (size_t)src->nelem;
    auto cp = [&](void* d, const void* s, size_t n) {
        return cudaMemcpyAsync(d, s, n, cudaMemcpyDeviceToDevice, src->st);
    };
    cudaError_t e = cudaSuccess;
    // both forms keep the same set of arrays; copy buffer for buffer
    auto copy_bufs = [&](auto& D, auto& S) {
        for (int v = 0; v < 4; ++v)
            for (int b = 0; b < 2; ++b) {
                if (e == cudaSuccess) e = cp(D.q[v][b], S.q[v][b], bytes);
                if (e == cudaSuccess) e = cp(D.H[v][b], S.H[v][b], bytes);
            }
        for (int b = 0; b < 2; ++b)
            for (int m = 0; m < 4; ++m)
                if (e == cudaSuccess) e = cp(D.mu[b][m], S.mu[b][m], bytes);
        for (int v = 1; v < 4; ++v)
            if (e == cudaSuccess) e = cp(D.pg[v], S.pg[v], bytes);
        if (e == cudaSuccess) e = cp(D.phi, S.phi, bytes);
    };
    if (src->mixed) copy_bufs(dst->b32, src->b32);
    else copy_bufs(dst->b64, src->b64);
    if (e == cudaSuccess) e = cp(dst->scal, src->scal, sizeof(double) * S_COUNT);
    if (e != cudaSuccess) return fail(src, PLLGPU_ECUDA);
    CK(cudaStreamSynchronize(src->st));
    dst->cur = src->cur;
    dst->rotated = src->rotated;
    dst->resync_c = src->resync_c;
    dst->timestep = src->timestep;
    return PLLGPU_OK;
}

int pllgpu_run_host(pllgpu_ctx* ctx, int nsteps, const double* c0, const double* u0, const double* v0,
                    const double* w0, double* c, double* u, double* v, double* w)
{
    if (!ctx) return PLLGPU_EINVAL;
    int e;
    if ((e = pllgpu_set_field(ctx, PLLGPU_C_NEW, c0)) || (e = pllgpu_set_field(ctx, PLLGPU_U_NEW, u0)) ||
        (e = pllgpu_set_field(ctx, PLLGPU_V_NEW, v0)) || (e = pllgpu_set_field(ctx, PLLGPU_W_NEW, w0)))
        return e;
    if ((e = pllgpu_start(ctx))) return e;
    if ((e = pllgpu_steps(ctx, nsteps))) return e;
    if ((c && (e = pllgpu_get_field(ctx, PLLGPU_C_NEW, c))) || (u && (e = pllgpu_get_field(ctx, PLLGPU_U_NEW, u))) ||
        (v && (e = pllgpu_get_field(ctx, PLLGPU_V_NEW, v))) || (w && (e = pllgpu_get_field(ctx, PLLGPU_W_NEW, w))))
        return e;
    return PLLGPU_OK;
}

int pllgpu_routine(pllgpu_ctx* ctx, int routine, const double* in, double* out)
{
    if (!ctx || routine < 0 || routine >= PLLGPU_NROUTINES) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    if (routine != PLLGPU_R_SUBSTEP)
        if (int e = materialize(ctx)) return e;
    int e = FORM_CALL(ctx, form_routine, ctx, routine, in, out);
    if (e) return e;
    if (int e2 = check_launch(ctx)) return e2;
    CK(cudaStreamSynchronize(ctx->st));
    return read_status(ctx);
}

int pllgpu_diagnostics(pllgpu_ctx* ctx, double* out4)
{
    if (!ctx || !out4) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    FORM_CALL(ctx, form_diag, ctx);
    if (int e = check_launch(ctx)) return e;
    CK(cudaMemcpyAsync(out4, ctx->diag + 3L * ni(ctx->Rg), sizeof(double) * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

int pllgpu_profile_steps(pllgpu_ctx* ctx, int nsteps, int maxk, char* names, double* total_ms, int* launches,
                         int* nk_out)
{
    // nsteps steps on the stream (no graph) with an event after every
    // launch; per kernel label: summed device time and launch count.
    // names: maxk slots of 32 chars.
    if (!ctx || nsteps < 1 || maxk < 1 || !names || !total_ms || !launches || !nk_out) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    ctx->profiling = true;
    ctx->ev_label.clear();
    mark(ctx, "start");  // a leading event so the first kernel has a start
    for (int s = 0; s < nsteps; ++s) enqueue_step_any(ctx);
    ctx->profiling = false;
    ctx->rotated = true;
    if (int e = check_launch(ctx)) return e;
    CK(cudaStreamSynchronize(ctx->st));
    int nk = 0;
    for (size_t i = 1; i < ctx->ev_label.size(); ++i) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev_pool[i - 1], ctx->ev_pool[i]));
        int slot = -1;
        for (int t = 0; t < nk; ++t)
            if (!std::strncmp(names + 32 * t, ctx->ev_label[i], 31)) slot = t;
        if (slot < 0) {
            if (nk >= maxk) continue;
            slot = nk++;
            std::strncpy(names + 32 * slot, ctx->ev_label[i], 31);
            names[32 * slot + 31] = 0;
            total_ms[slot] = 0.0;
            launches[slot] = 0;
        }
        total_ms[slot] += ms;
        launches[slot] += 1;
    }
    *nk_out = nk;
    ctx->ev_label.clear();
    return read_status(ctx);
}

void* pllgpu_stream(pllgpu_ctx* ctx) { return ctx ? (void*)ctx->st : nullptr; }

int pllgpu_sync(pllgpu_ctx* ctx)
{
    if (!ctx) return PLLGPU_EINVAL;
    CK(cudaStreamSynchronize(ctx->st));
    return read_status(ctx);
}

int pllgpu_status(const pllgpu_ctx* ctx) { return ctx ? ctx->err : PLLGPU_EINVAL; }

void pllgpu_clear_status(pllgpu_ctx* ctx)
{
    if (!ctx) return;
    ctx->err = PLLGPU_OK;
    cudaMemsetAsync(ctx->status, 0, sizeof(int), ctx->st);
    cudaStreamSynchronize(ctx->st);
}

double pllgpu_last_dt(pllgpu_ctx* ctx) { return ctx ? get_scalar(ctx, S_DT) : NAN; }
double pllgpu_timestep(const pllgpu_ctx* ctx) { return ctx ? ctx->timestep : NAN; }
double pllgpu_tval(pllgpu_ctx* ctx) { return ctx ? get_scalar(ctx, S_TVAL) : NAN; }
int pllgpu_kernels_per_step(const pllgpu_ctx* ctx) { return ctx ? ctx->launches_per_step : 0; }

int pllgpu_set_timestep(pllgpu_ctx* ctx, double ts)
{
    if (!ctx) return PLLGPU_EINVAL;
    ctx->timestep = ts;
    return set_scalar(ctx, S_TIMESTEP, ts);
}

int pllgpu_set_tval(pllgpu_ctx* ctx, double t)
{
    if (!ctx) return PLLGPU_EINVAL;
    return set_scalar(ctx, S_TVAL, t);
}

int pllgpu_acoef(pllgpu_ctx* ctx, int var, int which, double* abc9)
{
    if (!ctx || ctx->mixed || var < 0 || var > 3 || (which != 0 && which != 1) || !abc9) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    if (int e = materialize(ctx)) return e;
    const long ne = ctx->nelem;
    DevBuf buf;
    if (!buf.alloc(sizeof(double) * 9 * (size_t)ne)) return fail(ctx, PLLGPU_ECUDA);
    CK(cudaMemsetAsync(buf.p, 0, sizeof(double) * 9 * (size_t)ne, ctx->st));
    MuPtrs<double> m = which ? mu_new<double>(ctx) : mu_old<double>(ctx);
    const Rng& R = ctx->Rv[var];
    dim3 blk(32, 4), grd = box_grid(nk(R), nj(R), ni(R), blk);
    if (var == VC) k_acoef<VC><<<grd, blk, 0, ctx->st>>>(ctx->G, R, ctx->K, m, buf.d(), ne);
    else if (var == VU) k_acoef<VU><<<grd, blk, 0, ctx->st>>>(ctx->G, R, ctx->K, m, buf.d(), ne);
    else if (var == VV) k_acoef<VV><<<grd, blk, 0, ctx->st>>>(ctx->G, R, ctx->K, m, buf.d(), ne);
    else k_acoef<VW><<<grd, blk, 0, ctx->st>>>(ctx->G, R, ctx->K, m, buf.d(), ne);
    if (int e = check_launch(ctx)) return e;
    const Geo& G = ctx->G;
    for (int f = 0; f < 9; ++f)
        CK(cudaMemcpy2DAsync(abc9 + (long)f * G.NX * G.NY * G.NZ, sizeof(double) * G.NZ, buf.d() + (long)f * ne,
                             sizeof(double) * G.sy, sizeof(double) * G.NZ, (size_t)G.NX * G.NY,
                             cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

}  // extern "C"
