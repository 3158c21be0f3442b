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
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/pllcart3d_gpu.h"
#include "aux_kernels.cuh"
#include "common.cuh"
#include "dct_kernels.cuh"
#include "step_kernels.cuh"

using namespace pll;

namespace {

// RK3 (Wray) coefficients, global_variables.h:17-18
const double kRK1[3] = {(8.0 / 15.0), (5.0 / 12.0), (3.0 / 4.0)};
const double kRK2[3] = {(0.0), (-17.0 / 60.0), (-5.0 / 12.0)};

bool is_pow2(double h)
{
    int e;
    double m = std::frexp(h, &e);
    return m == 0.5;
}

// FFTW REDFT10 / REDFT01 as dense matrices T[k*n+j] (FFTW 3 manual,
// "1d Real-even DFTs (DCTs)"); the argument is reduced mod 4n exactly
void dct_matrix(int kind, int n, double* T)
{
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j) {
            long m;
            if (kind == 0) {
                m = ((long)(2 * j + 1) * (long)k) % (4L * n);
                T[(long)k * n + j] = 2.0 * std::cos(pi * (double)m / (2.0 * n));
            } else if (j == 0) {
                T[(long)k * n + j] = 1.0;
            } else {
                m = ((long)j * (long)(2 * k + 1)) % (4L * n);
                T[(long)k * n + j] = 2.0 * std::cos(pi * (double)m / (2.0 * n));
            }
        }
}

}  // namespace

struct pllgpu_ctx {
    pllgpu_params P;
    Geo G;
    Rng Rg, Rv[4];
    Consts K;
    Phys ph;
    int dev = 0;
    cudaStream_t st = nullptr;
    long nelem = 0;             // elements of one padded field
    double* q[4][2] = {};       // c, u, v, w : [role buffer]
    double* H[4][2] = {};
    double* mu[2][4] = {};      // [buffer][cell, xy, xz, yz]
    double* pg[4] = {};         // u, v, w at 1..3
    double* phi = nullptr;
    double* div = nullptr;
    double* S = nullptr;        // ADI right-hand side / eliminated rhs
    double* cc = nullptr;       // Thomas scratch
    double* dct1 = nullptr;     // compact nx*ny*nz buffers
    double* dct2 = nullptr;
    double *Ty = nullptr, *Tz = nullptr, *Tiy = nullptr, *Tiz = nullptr;
    double *lam_y = nullptr, *lam_z = nullptr;
    double* scal = nullptr;     // device scalars (S_*)
    int* status = nullptr;      // device sticky status bits
    double* work = nullptr;     // slope-parameter scratch
    int cur = 0;                // buffer index holding the "old" role
    bool rotated = false;       // fast steps ran: "new" roles are stale and
                                // logically equal to "old" (see materialize)
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    bool graphs_ready = false;
    double timestep = 0;
    int err = PLLGPU_OK;
    int launches_per_step = 0;
    int counting = 0;
    bool profiling = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<const char*> ev_label;
    std::vector<void*> allocs;

    double* q_old(int v) { return q[v][cur]; }
    double* q_new(int v) { return q[v][1 - cur]; }
    double* h_n(int v) { return H[v][1 - cur]; }
    double* h_nm1(int v) { return H[v][cur]; }
    MuPtrs<double> mu_old() { return {mu[cur][0], mu[cur][1], mu[cur][2], mu[cur][3]}; }
    MuPtrs<double> mu_new() { return {mu[1 - cur][0], mu[1 - cur][1], mu[1 - cur][2], mu[1 - cur][3]}; }
};

namespace {

int fail(pllgpu_ctx* c, int code)
{
    if (c && c->err == PLLGPU_OK) c->err = code;
    return code;
}

#define CK(call)                                                                     \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            std::fprintf(stderr, "pllgpu: %s failed: %s (%s:%d)\n", #call,           \
                         cudaGetErrorString(e_), __FILE__, __LINE__);                \
            return fail(ctx, PLLGPU_ECUDA);                                          \
        }                                                                            \
    } while (0)

// every kernel launch of the step goes through mark(): it counts launches
// and, in profiling mode, records an event after the launch so that the
// device time of each kernel is the gap to the previous event
void mark(pllgpu_ctx* ctx, const char* label);

double* dalloc(pllgpu_ctx* ctx, long n)
{
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, sizeof(double) * (size_t)(n > 0 ? n : 1));
    ctx->allocs.push_back(p);
    return (double*)p;
}

void mark(pllgpu_ctx* ctx, const char* label)
{
    ctx->counting++;
    if (!ctx->profiling) return;
    const size_t i = ctx->ev_label.size();
    if (i >= ctx->ev_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ctx->ev_pool.push_back(e);
    }
    cudaEventRecord(ctx->ev_pool[i], ctx->st);
    ctx->ev_label.push_back(label);
}

dim3 box_grid(int nk, int nj, int ni, dim3 blk)
{
    return dim3((nk + blk.x - 1) / blk.x, (nj + blk.y - 1) / blk.y, ni);
}

int ni(const Rng& r) { return r.ie - r.is + 1; }
int nj(const Rng& r) { return r.je - r.js + 1; }
int nk(const Rng& r) { return r.ke - r.ks + 1; }

// ---- stage launchers -------------------------------------------------------

template <int VAR>
void launch_explicit(pllgpu_ctx* ctx, const double* un, const double* vn, const double* wn,
                     double g, double r)
{
    const Rng& R = ctx->Rv[VAR];
    ExplicitArgs<double> A;
    A.q = ctx->q_old(VAR);
    A.un = un;
    A.vn = vn;
    A.wn = wn;
    A.mu = ctx->mu_old();
    A.cn = ctx->q_new(VC);
    A.pg = VAR == VC ? nullptr : ctx->pg[VAR];
    A.Hm = ctx->h_nm1(VAR);
    A.H = ctx->h_n(VAR);
    A.S = ctx->S;
    A.scal = ctx->scal;
    A.g = g;
    A.r = r;
    A.alpha = g + r;
    dim3 blk(32, 4);
    k_explicit<VAR, double><<<box_grid(nk(R), nj(R), ni(R), blk), blk, 0, ctx->st>>>(ctx->G, R, ctx->K, A);
    mark(ctx, VAR == VC ? "explicit_c" : VAR == VU ? "explicit_u" : VAR == VV ? "explicit_v" : "explicit_w");
}

template <int VAR>
void launch_implicit(pllgpu_ctx* ctx, double g, double r)
{
    const Rng& R = ctx->Rv[VAR];
    const double alpha = g + r;
    MuPtrs<double> mn = ctx->mu_new();
    XsweepArgs<double> X;
    X.mu = mn;
    X.q = ctx->q_old(VAR);
    X.qn = ctx->q_new(VAR);
    X.H = ctx->h_n(VAR);
    X.Hm = ctx->h_nm1(VAR);
    X.S = ctx->S;
    X.cc = ctx->cc;
    X.scal = ctx->scal;
    X.g = g;
    X.r = r;
    X.alpha = alpha;
    k_line_pf<VAR, 1, double><<<dim3((nk(R) + 63) / 64, ni(R)), 64, 0, ctx->st>>>(ctx->G, R, ctx->K, X);
    mark(ctx, VAR == VC ? "adi_y_c" : VAR == VU ? "adi_y_u" : VAR == VV ? "adi_y_v" : "adi_y_w");
    {
        constexpr size_t smem = adi_z_smem_bytes<VAR, double>();
        k_adi_z_tiled<VAR, double><<<dim3((nj(R) + 127) / 128, ni(R)), 128, smem, ctx->st>>>(
            ctx->G, R, ctx->K, mn, ctx->S, ctx->cc, ctx->scal, alpha);
    }
    mark(ctx, VAR == VC ? "adi_z_c" : VAR == VU ? "adi_z_u" : VAR == VV ? "adi_z_v" : "adi_z_w");
    k_line_pf<VAR, 0, double><<<dim3((nk(R) + 63) / 64, nj(R)), 64, 0, ctx->st>>>(ctx->G, R, ctx->K, X);
    mark(ctx, VAR == VC ? "adi_x_c" : VAR == VU ? "adi_x_u" : VAR == VV ? "adi_x_v" : "adi_x_w");
}

void launch_viscosity(pllgpu_ctx* ctx, const double* cn, MuPtrs<double> m, int law = -1)
{
    dim3 blk(32, 4);
    k_viscosity<double><<<box_grid(ctx->G.NZ, ctx->G.NY, ni(ctx->Rg) + 2, blk), blk, 0, ctx->st>>>(
        ctx->G, ctx->Rg, ctx->K, law < 0 ? ctx->P.nmvp : law, cn, (double*)m.cell, (double*)m.xy, (double*)m.xz,
        (double*)m.yz, ctx->scal);
    mark(ctx, "viscosity");
}

void launch_gemm(pllgpu_ctx* ctx, const GemmDesc& d, const double* A, const double* B, double* C)
{
    dim3 grid((d.N + 63) / 64, (d.M + 63) / 64, d.batch);
    if (ctx->P.exact_dct)
        k_gemm_seq<double><<<grid, 256, 0, ctx->st>>>(d, A, B, C);
    else
        k_gemm_dmma<<<grid, 256, 0, ctx->st>>>(d, A, B, C);
    mark(ctx, "dct_gemm");
}

// phisolver_dct after its right-hand side is in dct1 (compact [x][y][z])
void launch_poisson(pllgpu_ctx* ctx)
{
    const int nx = ctx->G.nx, ny = ctx->G.ny, nz = ctx->G.nz;
    const long N = (long)ny * nz;
    GemmDesc d{};
    // forward, y pass: dct2[x][ky][z] = sum_y Ty[ky][y] dct1[x][y][z]
    d = GemmDesc{ny, nz, ny, nx, 0, ny, 1, N, nz, 1, N, nz, 1, 0.0, 0};
    launch_gemm(ctx, d, ctx->Ty, ctx->dct1, ctx->dct2);
    // forward, z pass: dct1[x][ky][kz] = sum_z dct2[x][ky][z] Tz[kz][z]
    d = GemmDesc{ny, nz, nz, nx, N, nz, 1, 0, 1, nz, N, nz, 1, 0.0, 0};
    launch_gemm(ctx, d, ctx->dct2, ctx->Tz, ctx->dct1);
    // x-tridiagonal per mode, in place in dct1 (dct2 as scratch)
    k_poisson_x<double><<<(int)((N + 127) / 128), 128, 0, ctx->st>>>(nx, ny, nz, ctx->K, ctx->lam_y,
                                                                    ctx->lam_z, ctx->dct1, ctx->dct2);
    mark(ctx, "poisson_x");
    // inverse, y pass: dct2[x][y][kz] = sum_ky Tiy[y][ky] dct1[x][ky][kz]
    d = GemmDesc{ny, nz, ny, nx, 0, ny, 1, N, nz, 1, N, nz, 1, 0.0, 0};
    launch_gemm(ctx, d, ctx->Tiy, ctx->dct1, ctx->dct2);
    // inverse, z pass into phi's interior, divided by 4*ny*nz
    const double four_n = (double)(4 * N);
    d = GemmDesc{ny, nz, nz, nx, N, nz, 1, 0, 1, nz, ctx->G.sx, ctx->G.sy, 1,
                 is_pow2(four_n) ? 1.0 / four_n : four_n, is_pow2(four_n) ? 1 : 2};
    double* phi0 = ctx->phi + (long)ctx->Rg.is * ctx->G.sx + (long)ctx->Rg.js * ctx->G.sy + ctx->Rg.ks;
    launch_gemm(ctx, d, ctx->dct2, ctx->Tiz, phi0);
}

void launch_phi_ghosts(pllgpu_ctx* ctx)
{
    const Rng& R = ctx->Rg;
    k_phi_ghosts<0, double><<<dim3((nj(R) + 127) / 128, ni(R)), 128, 0, ctx->st>>>(ctx->G, R, ctx->phi);
    mark(ctx, "phi_ghosts");
    k_phi_ghosts<1, double><<<dim3((nk(R) + 127) / 128, ni(R)), 128, 0, ctx->st>>>(ctx->G, R, ctx->phi);
    mark(ctx, "phi_ghosts");
    k_phi_ghosts<2, double><<<dim3((nk(R) + 127) / 128, nj(R)), 128, 0, ctx->st>>>(ctx->G, R, ctx->phi);
    mark(ctx, "phi_ghosts");
}

void launch_project(pllgpu_ctx* ctx, double alpha, int correct, int ghosts, int pgu)
{
    ProjectArgs<double> A;
    A.u = ctx->q_new(VU);
    A.v = ctx->q_new(VV);
    A.w = ctx->q_new(VW);
    A.pgu = ctx->pg[VU];
    A.pgv = ctx->pg[VV];
    A.pgw = ctx->pg[VW];
    A.phi = ctx->phi;
    A.mu = ctx->mu_new();
    A.scal = ctx->scal;
    A.alpha = alpha;
    A.do_correct = correct;
    A.do_ghosts = ghosts;
    A.do_pg = pgu;
    dim3 blk(32, 4);
    k_project<double><<<box_grid(nk(ctx->Rg), nj(ctx->Rg), ni(ctx->Rg) + 1, blk), blk, 0, ctx->st>>>(
        ctx->G, ctx->Rg, ctx->Rv[VU], ctx->Rv[VV], ctx->Rv[VW], ctx->K, A);
    mark(ctx, "project");
}

void launch_div(pllgpu_ctx* ctx, int mode, double alpha)
{
    dim3 blk(32, 4);
    k_div_rhs<double><<<box_grid(nk(ctx->Rg), nj(ctx->Rg), ni(ctx->Rg), blk), blk, 0, ctx->st>>>(
        ctx->G, ctx->Rg, ctx->K, ctx->q_new(VU), ctx->q_new(VV), ctx->q_new(VW), ctx->div, ctx->div,
        ctx->dct1, ctx->scal, alpha, mode);
    mark(ctx, "div_rhs");
}

void launch_flux(pllgpu_ctx* ctx)
{
    k_flux<double><<<1, 512, sizeof(double) * 2 * ctx->G.NY, ctx->st>>>(ctx->G, ctx->Rv[VU], ctx->K,
                                                                         ctx->q_new(VU), ctx->scal);
    mark(ctx, "flux");
}

void launch_bulk(pllgpu_ctx* ctx)
{
    k_bulk_velo<double><<<1, 1024, 0, ctx->st>>>(ctx->G, ctx->Rg, ctx->q_old(VU), ctx->scal);
    mark(ctx, "bulk_velo");
}

void launch_cfl(pllgpu_ctx* ctx)
{
    dim3 blk(32, 8);
    k_cfl<double><<<box_grid(nk(ctx->Rg), nj(ctx->Rg), ni(ctx->Rg), blk), blk, 0, ctx->st>>>(
        ctx->G, ctx->Rg, ctx->K, ctx->q_old(VU), ctx->q_old(VV), ctx->q_old(VW), ctx->scal,
        ctx->status);
    mark(ctx, "cfl");
    k_dt<<<1, 1, 0, ctx->st>>>(ctx->K, ctx->scal);
    mark(ctx, "dt");
}

// one RK3-CN substep of the fast path, pllcart3d.c:164-194
void enqueue_substep(pllgpu_ctx* ctx, int rk)
{
    const double g = kRK1[rk], r = kRK2[rk], alpha = g + r;
    launch_bulk(ctx);
    // concentration: advected by u->new == u->old
    launch_explicit<VC>(ctx, ctx->q_old(VU), ctx->q_old(VV), ctx->q_old(VW), g, r);
    launch_implicit<VC>(ctx, g, r);
    launch_viscosity(ctx, ctx->q_new(VC), ctx->mu_new());
    launch_explicit<VU>(ctx, ctx->q_old(VU), ctx->q_old(VV), ctx->q_old(VW), g, r);
    launch_implicit<VU>(ctx, g, r);
    launch_explicit<VV>(ctx, ctx->q_old(VU), ctx->q_old(VV), ctx->q_old(VW), g, r);
    launch_implicit<VV>(ctx, g, r);
    launch_explicit<VW>(ctx, ctx->q_old(VU), ctx->q_old(VV), ctx->q_old(VW), g, r);
    launch_implicit<VW>(ctx, g, r);
    // update_velo_boundary (L182) writes only ghost entries that nothing
    // reads before update_veloghost_points (L189) rewrites them; skipped
    launch_flux(ctx);
    launch_div(ctx, 0, alpha);
    launch_poisson(ctx);
    launch_phi_ghosts(ctx);
    launch_project(ctx, alpha, 1, 1, 1);
    ctx->cur ^= 1;  // update_old_*: roles swap
}

void enqueue_step(pllgpu_ctx* ctx)
{
    launch_cfl(ctx);
    for (int rk = 0; rk < 3; ++rk) enqueue_substep(ctx, rk);
}

__global__ void k_tval(double* scal, double a0, double a1, double a2)
{
    // tval += (gamma+rho) dt per substep, pllcart3d.c:166
    const double dt = scal[S_DT];
    double t = scal[S_TVAL];
    t = t + a0 * dt;
    t = t + a1 * dt;
    t = t + a2 * dt;
    scal[S_TVAL] = t;
}

int set_scalar(pllgpu_ctx* ctx, int slot, double v)
{
    CK(cudaMemcpyAsync(ctx->scal + slot, &v, sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

double get_scalar(pllgpu_ctx* ctx, int slot)
{
    double v = NAN;
    if (cudaMemcpyAsync(&v, ctx->scal + slot, sizeof(double), cudaMemcpyDeviceToHost, ctx->st) != cudaSuccess ||
        cudaStreamSynchronize(ctx->st) != cudaSuccess)
        fail(ctx, PLLGPU_ECUDA);
    return v;
}

int check_launch(pllgpu_ctx* ctx)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "pllgpu: kernel launch failed: %s\n", cudaGetErrorString(e));
        return fail(ctx, PLLGPU_ECUDA);
    }
    return PLLGPU_OK;
}

int read_status(pllgpu_ctx* ctx)
{
    int s = 0;
    CK(cudaMemcpyAsync(&s, ctx->status, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (s & ST_NAN) return fail(ctx, PLLGPU_ENAN);
    if (s & ST_NOCONV) return fail(ctx, PLLGPU_ENOCONV);
    if (s & ST_BOUNDS) return fail(ctx, PLLGPU_EBOUNDS);
    return PLLGPU_OK;
}

int build_graphs(pllgpu_ctx* ctx)
{
    for (int t = 0; t < 2; ++t) {
        const int c0 = ctx->cur;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
        ctx->counting = 0;
        enqueue_step(ctx);
        k_tval<<<1, 1, 0, ctx->st>>>(ctx->scal, kRK1[0] + kRK2[0], kRK1[1] + kRK2[1], kRK1[2] + kRK2[2]);
        mark(ctx, "tval");
        CK(cudaStreamEndCapture(ctx->st, &g));
        ctx->launches_per_step = ctx->counting;
        CK(cudaGraphInstantiate(&ctx->gexec[c0], g, 0));
        cudaGraphDestroy(g);
        // cur flipped once by the three substeps
    }
    ctx->graphs_ready = true;
    return PLLGPU_OK;
}

}  // namespace

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
    if (p->precision != PLLGPU_FP64) return nullptr;
    pllgpu_ctx* ctx = new pllgpu_ctx();
    ctx->P = *p;
    ctx->dev = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess) {
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
    bool ok = true;
    for (int v = 0; v < 4 && ok; ++v)
        for (int b = 0; b < 2 && ok; ++b) {
            ok = (c->q[v][b] = dalloc(c, c->nelem)) && (c->H[v][b] = dalloc(c, c->nelem));
        }
    for (int b = 0; b < 2 && ok; ++b)
        for (int m = 0; m < 4 && ok; ++m) ok = (c->mu[b][m] = dalloc(c, c->nelem)) != nullptr;
    for (int v = 1; v < 4 && ok; ++v) ok = (c->pg[v] = dalloc(c, c->nelem)) != nullptr;
    const long ncell = (long)p->nx * p->ny * p->nz;
    ok = ok && (c->phi = dalloc(c, c->nelem)) && (c->div = dalloc(c, c->nelem)) &&
         (c->S = dalloc(c, c->nelem)) && (c->cc = dalloc(c, c->nelem)) &&
         (c->dct1 = dalloc(c, ncell)) && (c->dct2 = dalloc(c, ncell)) &&
         (c->Ty = dalloc(c, (long)p->ny * p->ny)) && (c->Tz = dalloc(c, (long)p->nz * p->nz)) &&
         (c->Tiy = dalloc(c, (long)p->ny * p->ny)) && (c->Tiz = dalloc(c, (long)p->nz * p->nz)) &&
         (c->lam_y = dalloc(c, p->ny)) && (c->lam_z = dalloc(c, p->nz)) &&
         (c->scal = dalloc(c, S_COUNT)) && (c->work = dalloc(c, 2L * (p->nx + 8)));
    if (ok) {
        void* sp = nullptr;
        ok = cudaMalloc(&sp, sizeof(int)) == cudaSuccess;
        if (ok) {
            cudaMemset(sp, 0, sizeof(int));
            c->allocs.push_back(sp);
            c->status = (int*)sp;
        }
    }
    if (!ok) {
        pllgpu_destroy(ctx);
        return nullptr;
    }
    // kernels above the 48 KB default of dynamic shared memory
    cudaFuncSetAttribute(k_adi_z_tiled<VC, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)adi_z_smem_bytes<VC, double>());
    cudaFuncSetAttribute(k_adi_z_tiled<VU, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)adi_z_smem_bytes<VU, double>());
    cudaFuncSetAttribute(k_adi_z_tiled<VV, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)adi_z_smem_bytes<VV, double>());
    cudaFuncSetAttribute(k_adi_z_tiled<VW, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)adi_z_smem_bytes<VW, double>());
    // DCT matrices and Poisson eigenvalues (phisolver_dct L2050-2051)
    {
        const double PI = 4.0 * std::atan(1.0);
        std::vector<double> T((size_t)std::max(p->ny, p->nz) * std::max(p->ny, p->nz));
        dct_matrix(0, p->ny, T.data());
        cudaMemcpy(c->Ty, T.data(), sizeof(double) * p->ny * p->ny, cudaMemcpyHostToDevice);
        dct_matrix(0, p->nz, T.data());
        cudaMemcpy(c->Tz, T.data(), sizeof(double) * p->nz * p->nz, cudaMemcpyHostToDevice);
        dct_matrix(1, p->ny, T.data());
        cudaMemcpy(c->Tiy, T.data(), sizeof(double) * p->ny * p->ny, cudaMemcpyHostToDevice);
        dct_matrix(1, p->nz, T.data());
        cudaMemcpy(c->Tiz, T.data(), sizeof(double) * p->nz * p->nz, cudaMemcpyHostToDevice);
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

// After fast steps the reference's state has new == old (update_old_*
// copies); the ping-pong buffers hold a stale "new".  Reads of new-role
// fields then see the old-role buffer; writes first copy old -> new.
static bool is_new_role(int f)
{
    return f == PLLGPU_C_NEW || f == PLLGPU_C_HN || f == PLLGPU_U_NEW || f == PLLGPU_U_HN ||
           f == PLLGPU_V_NEW || f == PLLGPU_V_HN || f == PLLGPU_W_NEW || f == PLLGPU_W_HN ||
           (f >= PLLGPU_MU_NEW_CELL && f <= PLLGPU_MU_NEW_YZ);
}

static int new_to_old(int f)
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

static int materialize(pllgpu_ctx* ctx)
{
    if (!ctx->rotated) return PLLGPU_OK;
    const size_t bytes = sizeof(double) * (size_t)ctx->nelem;
    for (int v = 0; v < 4; ++v) {
        CK(cudaMemcpyAsync(ctx->q_new(v), ctx->q_old(v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->h_n(v), ctx->h_nm1(v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->mu[1 - ctx->cur][v], ctx->mu[ctx->cur][v], bytes, cudaMemcpyDeviceToDevice,
                           ctx->st));
    }
    CK(cudaStreamSynchronize(ctx->st));
    ctx->rotated = false;
    return PLLGPU_OK;
}

static double* field_ptr_raw(pllgpu_ctx* ctx, int f);

static double* field_ptr(pllgpu_ctx* ctx, int f, bool for_write)
{
    if (f < 0 || f >= PLLGPU_NFIELDS) return nullptr;
    if (ctx->rotated && is_new_role(f)) {
        if (!for_write) return field_ptr_raw(ctx, new_to_old(f));
        if (materialize(ctx)) return nullptr;
    }
    return field_ptr_raw(ctx, f);
}

static double* field_ptr_raw(pllgpu_ctx* ctx, int f)
{
    if (f < 0 || f >= PLLGPU_NFIELDS) return nullptr;
    if (f <= PLLGPU_C_HNM1) {
        const int r = f - PLLGPU_C_OLD;
        return r == 0 ? ctx->q_old(VC) : r == 1 ? ctx->q_new(VC) : r == 2 ? ctx->h_n(VC) : ctx->h_nm1(VC);
    }
    if (f <= PLLGPU_W_PG) {
        const int v = 1 + (f - PLLGPU_U_OLD) / 5, r = (f - PLLGPU_U_OLD) % 5;
        return r == 0 ? ctx->q_old(v) : r == 1 ? ctx->q_new(v) : r == 2 ? ctx->h_n(v)
             : r == 3 ? ctx->h_nm1(v) : ctx->pg[v];
    }
    if (f <= PLLGPU_MU_OLD_YZ) return ctx->mu[ctx->cur][f - PLLGPU_MU_OLD_CELL];
    if (f <= PLLGPU_MU_NEW_YZ) return ctx->mu[1 - ctx->cur][f - PLLGPU_MU_NEW_CELL];
    if (f == PLLGPU_PHI) return ctx->phi;
    return ctx->div;
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
    double* d = field_ptr(ctx, f, true);
    if (!d) return fail(ctx, PLLGPU_EINVAL);
    const Geo& G = ctx->G;
    CK(cudaMemcpy2DAsync(d, sizeof(double) * G.sy, host, sizeof(double) * G.NZ, sizeof(double) * G.NZ,
                         (size_t)G.NX * G.NY, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

int pllgpu_get_field(pllgpu_ctx* ctx, int f, double* host)
{
    if (!ctx || !host) return PLLGPU_EINVAL;
    double* d = field_ptr(ctx, f, false);
    if (!d) return fail(ctx, PLLGPU_EINVAL);
    const Geo& G = ctx->G;
    CK(cudaMemcpy2DAsync(host, sizeof(double) * G.NZ, d, sizeof(double) * G.sy, sizeof(double) * G.NZ,
                         (size_t)G.NX * G.NY, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PLLGPU_OK;
}

int pllgpu_device_field(pllgpu_ctx* ctx, int f, double** dptr, long* si, long* sj)
{
    if (!ctx) return PLLGPU_EINVAL;
    double* d = field_ptr(ctx, f, true);
    if (!d) return PLLGPU_EINVAL;
    if (dptr) *dptr = d;
    if (si) *si = ctx->G.sx;
    if (sj) *sj = ctx->G.sy;
    return PLLGPU_OK;
}

int pllgpu_start(pllgpu_ctx* ctx)
{
    if (!ctx) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    if (int e = materialize(ctx)) return e;
    const size_t bytes = sizeof(double) * (size_t)ctx->nelem;
    // update_ghost_points (L81) on the initial velocities; phi is zero
    launch_project(ctx, 0.0, 0, 1, 0);
    // update_old_conc / update_old_velo (L82-83): both buffers equal
    for (int v = 0; v < 4; ++v) {
        CK(cudaMemcpyAsync(ctx->q_old(v), ctx->q_new(v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->h_nm1(v), ctx->h_n(v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
    }
    if (ctx->P.nmvp) {
        const double PI = 4.0 * std::atan(1.0);
        k_slope_parameter<<<1, 1, 0, ctx->st>>>(ctx->G, ctx->Rg, ctx->P.Y1, ctx->P.Z1, ctx->G.dy, ctx->G.dz,
                                                ctx->P.Vratio, ctx->P.Mum, ctx->P.Lambda, PI,
                                                ctx->q_new(VC), ctx->scal, ctx->status, ctx->work);
    }
    // calculate_viscosity(c->old, mu_old), L142
    launch_viscosity(ctx, ctx->q_old(VC), ctx->mu_old());
    if (int e = check_launch(ctx)) return e;
    CK(cudaStreamSynchronize(ctx->st));
    set_scalar(ctx, S_TVAL, 0.0);
    return read_status(ctx);
}

int pllgpu_steps(pllgpu_ctx* ctx, int nsteps)
{
    if (!ctx || nsteps < 0) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
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
            enqueue_step(ctx);
            k_tval<<<1, 1, 0, ctx->st>>>(ctx->scal, kRK1[0] + kRK2[0], kRK1[1] + kRK2[1], kRK1[2] + kRK2[2]);
            mark(ctx, "tval");
            ctx->launches_per_step = ctx->counting;
            if (int e = check_launch(ctx)) return e;
        }
    }
    if (nsteps > 0) ctx->rotated = true;
    CK(cudaStreamSynchronize(ctx->st));
    return read_status(ctx);
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
    double dt = in ? in[0] : 0.0, g = in ? in[1] : 0.0, r = in ? in[2] : 0.0, vb = in ? in[3] : 0.0;
    const double alpha = g + r;
    const size_t bytes = sizeof(double) * (size_t)ctx->nelem;
    switch (routine) {
    case PLLGPU_R_CONCENTRATION:
        if (set_scalar(ctx, S_DT, dt) || set_scalar(ctx, S_VBULK, vb)) return ctx->err;
        launch_explicit<VC>(ctx, ctx->q_new(VU), ctx->q_new(VV), ctx->q_new(VW), g, r);
        launch_implicit<VC>(ctx, g, r);
        break;
    case PLLGPU_R_VISCOSITY_NEW:
        launch_viscosity(ctx, ctx->q_new(VC), ctx->mu_new());
        break;
    case PLLGPU_R_XMOM:
    case PLLGPU_R_YMOM:
    case PLLGPU_R_ZMOM:
        if (set_scalar(ctx, S_DT, dt) || set_scalar(ctx, S_VBULK, vb)) return ctx->err;
        if (routine == PLLGPU_R_XMOM) {
            launch_explicit<VU>(ctx, ctx->q_old(VU), ctx->q_old(VV), ctx->q_old(VW), g, r);
            launch_implicit<VU>(ctx, g, r);
        } else if (routine == PLLGPU_R_YMOM) {
            launch_explicit<VV>(ctx, ctx->q_old(VU), ctx->q_old(VV), ctx->q_old(VW), g, r);
            launch_implicit<VV>(ctx, g, r);
        } else {
            launch_explicit<VW>(ctx, ctx->q_old(VU), ctx->q_old(VV), ctx->q_old(VW), g, r);
            launch_implicit<VW>(ctx, g, r);
        }
        break;
    case PLLGPU_R_VELO_GHOSTS:
        launch_project(ctx, 0.0, 0, 1, 0);
        break;
    case PLLGPU_R_DIVERGENCE:
        launch_div(ctx, 1, 0.0);
        break;
    case PLLGPU_R_PHISOLVER:
        if (set_scalar(ctx, S_DT, dt)) return ctx->err;
        launch_div(ctx, 2, alpha);
        launch_poisson(ctx);
        break;
    case PLLGPU_R_PHI_GHOSTS:
        launch_phi_ghosts(ctx);
        break;
    case PLLGPU_R_VELO_CORRECTION:
        if (set_scalar(ctx, S_DT, dt)) return ctx->err;
        launch_flux(ctx);
        launch_project(ctx, alpha, 1, 0, 0);
        break;
    case PLLGPU_R_PRESSURE_GRADIENT:
        if (set_scalar(ctx, S_DT, dt)) return ctx->err;
        launch_project(ctx, alpha, 0, 0, 1);
        break;
    case PLLGPU_R_ROTATE:
        for (int v = 0; v < 4; ++v) {
            CK(cudaMemcpyAsync(ctx->q_old(v), ctx->q_new(v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
            CK(cudaMemcpyAsync(ctx->h_nm1(v), ctx->h_n(v), bytes, cudaMemcpyDeviceToDevice, ctx->st));
            CK(cudaMemcpyAsync(ctx->mu[ctx->cur][v], ctx->mu[1 - ctx->cur][v], bytes, cudaMemcpyDeviceToDevice,
                               ctx->st));
        }
        break;
    case PLLGPU_R_BULK_VELO:
        launch_bulk(ctx);
        if (out) out[0] = get_scalar(ctx, S_VBULK);
        break;
    case PLLGPU_R_FIND_CFL:
        // find_cfl's own return value CFLmax/max (before the Timestep clip)
        launch_cfl(ctx);
        if (out) out[0] = get_scalar(ctx, S_CFLDT);
        break;
    case PLLGPU_R_VISCOSITY_EXP:
        launch_viscosity(ctx, ctx->q_new(VC), ctx->mu_new(), 0);
        break;
    case PLLGPU_R_VISCOSITY_NMVP: {
        // coefficients of calculate_viscosity_nmvp (pllcart3d.c:895-900)
        const double cm = dt, PI = 4.0 * std::atan(1.0), M = ctx->P.Vratio;
        const double alpha = std::exp(M), mum = ctx->P.Mum * alpha;
        const double psi0 = std::asin(alpha / mum), psi1 = PI - std::asin(1 / mum);
        const double etam = (PI / 2 - psi0) / (psi1 - psi0);
        const double a = ((1 - cm) - etam) / ((1 - cm) * (etam - 1));
        if (set_scalar(ctx, S_CM, cm) || set_scalar(ctx, S_MUM, mum) || set_scalar(ctx, S_PSI0, psi0) ||
            set_scalar(ctx, S_PSI1, psi1) || set_scalar(ctx, S_NMVA, a))
            return ctx->err;
        launch_viscosity(ctx, ctx->q_new(VC), ctx->mu_new(), 1);
        break;
    }
    case PLLGPU_R_SLOPE_PARAMETER: {
        const double PI = 4.0 * std::atan(1.0);
        k_slope_parameter<<<1, 1, 0, ctx->st>>>(ctx->G, ctx->Rg, ctx->P.Y1, ctx->P.Z1, ctx->G.dy, ctx->G.dz,
                                                ctx->P.Vratio, ctx->P.Mum, ctx->P.Lambda, PI, ctx->q_new(VC),
                                                ctx->scal, ctx->status, ctx->work);
        mark(ctx, "slope_parameter");
        if (out) out[0] = get_scalar(ctx, S_CM);
        break;
    }
    case PLLGPU_R_SUBSTEP: {
        const int rk = (int)g;
        if (rk < 0 || rk > 2) return fail(ctx, PLLGPU_EINVAL);
        if (set_scalar(ctx, S_DT, dt)) return ctx->err;
        enqueue_substep(ctx, rk);
        ctx->rotated = true;
        break;
    }
    default:
        return fail(ctx, PLLGPU_EINVAL);
    }
    if (int e = check_launch(ctx)) return e;
    CK(cudaStreamSynchronize(ctx->st));
    return read_status(ctx);
}

int pllgpu_profile_steps(pllgpu_ctx* ctx, int nsteps, int maxk, char* names, double* total_ms,
                         int* launches, int* nk_out)
{
    // nsteps steps on the stream (no graph) with an event after every
    // launch; per kernel label: summed device time and launch count.
    // names: maxk slots of 32 chars.
    if (!ctx || nsteps < 1 || maxk < 1 || !names || !total_ms || !launches || !nk_out) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    ctx->profiling = true;
    ctx->ev_label.clear();
    const size_t first = 0;
    // a leading event so the first kernel has a start
    mark(ctx, "start");
    for (int s = 0; s < nsteps; ++s) {
        enqueue_step(ctx);
        k_tval<<<1, 1, 0, ctx->st>>>(ctx->scal, kRK1[0] + kRK2[0], kRK1[1] + kRK2[1], kRK1[2] + kRK2[2]);
        mark(ctx, "tval");
    }
    ctx->profiling = false;
    ctx->rotated = true;
    if (int e = check_launch(ctx)) return e;
    CK(cudaStreamSynchronize(ctx->st));
    int nk = 0;
    for (size_t i = first + 1; i < ctx->ev_label.size(); ++i) {
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

}  // extern "C"

// ---------------------------------------------------------------------------
// stand-alone batched primitives on host buffers (drop-in pll_tridiag and
// fdct_3d / idct_3d); the default CUDA device and stream
// ---------------------------------------------------------------------------
namespace {

// pll_tridiag's one-rank arithmetic on N contiguous systems of length n
__global__ void k_tridiag_batch(int N, int n, const double* __restrict__ a, double* __restrict__ b,
                                double* __restrict__ c, double* __restrict__ r)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const long o = (long)s * n;
    b[o] = b[o] - 0.0 * a[o];
    c[o] = c[o] / b[o];
    r[o] = (r[o] - 0.0 * a[o]) / b[o];
    for (int i = 1; i < n; ++i) {
        b[o + i] = (b[o + i] - c[o + i - 1] * a[o + i]);
        c[o + i] = c[o + i] / b[o + i];
        r[o + i] = (r[o + i] - r[o + i - 1] * a[o + i]) / b[o + i];
    }
    r[o + n - 1] = r[o + n - 1] - c[o + n - 1] * 0.0;
    for (int i = n - 2; i >= 0; --i) r[o + i] = r[o + i] - c[o + i] * r[o + i + 1];
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    bool alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 8) == cudaSuccess; }
    double* d() { return (double*)p; }
};

}  // namespace

extern "C" int pllgpu_tridiag_batch(int N, int n, const double* a, double* b, double* c, double* r)
{
    if (N < 0 || n < 1 || !a || !b || !c || !r) return PLLGPU_EINVAL;
    if (N == 0) return PLLGPU_OK;
    const size_t bytes = sizeof(double) * (size_t)N * n;
    DevBuf da, db, dc, dr;
    if (!da.alloc(bytes) || !db.alloc(bytes) || !dc.alloc(bytes) || !dr.alloc(bytes)) return PLLGPU_ECUDA;
    if (cudaMemcpy(da.p, a, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(db.p, b, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dc.p, c, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dr.p, r, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    k_tridiag_batch<<<(N + 127) / 128, 128>>>(N, n, da.d(), db.d(), dc.d(), dr.d());
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(b, db.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(c, dc.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(r, dr.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return PLLGPU_ECUDA;
    return PLLGPU_OK;
}

extern "C" int pllgpu_dct2d_batch(int kind, int n0, int n1, int howmany, const double* in, double* out)
{
    if ((kind != 0 && kind != 1) || n0 < 1 || n1 < 1 || howmany < 0 || !in || !out) return PLLGPU_EINVAL;
    if (howmany == 0) return PLLGPU_OK;
    const long per = (long)n0 * n1;
    const size_t bytes = sizeof(double) * (size_t)per * howmany;
    std::vector<double> T0((size_t)n0 * n0), T1((size_t)n1 * n1);
    dct_matrix(kind, n0, T0.data());
    dct_matrix(kind, n1, T1.data());
    DevBuf dT0, dT1, dx, dtmp, dy;
    if (!dT0.alloc(sizeof(double) * T0.size()) || !dT1.alloc(sizeof(double) * T1.size()) || !dx.alloc(bytes) ||
        !dtmp.alloc(bytes) || !dy.alloc(bytes))
        return PLLGPU_ECUDA;
    if (cudaMemcpy(dT0.p, T0.data(), sizeof(double) * T0.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dT1.p, T1.data(), sizeof(double) * T1.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dx.p, in, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    // along the fast dimension: tmp[t][r][k] = sum_j T1[k][j] x[t][r][j]
    GemmDesc d1{n0, n1, n1, howmany, per, n1, 1, 0, 1, n1, per, n1, 1, 0.0, 0};
    k_gemm_seq<double><<<dim3((n1 + 63) / 64, (n0 + 63) / 64, howmany), 256>>>(d1, dx.d(), dT1.d(), dtmp.d());
    // along the slow dimension: y[t][k][c] = sum_r T0[k][r] tmp[t][r][c]
    GemmDesc d2{n0, n1, n0, howmany, 0, n0, 1, per, n1, 1, per, n1, 1, 0.0, 0};
    k_gemm_seq<double><<<dim3((n1 + 63) / 64, (n0 + 63) / 64, howmany), 256>>>(d2, dT0.d(), dtmp.d(), dy.d());
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(out, dy.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return PLLGPU_ECUDA;
    return PLLGPU_OK;
}

// ---------------------------------------------------------------------------
// coefficient export, setters and stand-alone primitives of the drop-in layer
// ---------------------------------------------------------------------------
namespace {

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

__global__ void k_weno_batch(int n, const double* __restrict__ v5, double* __restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double* v = v5 + 5L * t;
    out[t] = weno5<double>(v[0], v[1], v[2], v[3], v[4]);
}

// tridiag_1rhs on N contiguous systems; c' in scratch cc
__global__ void k_tridiag_1rhs_batch(int N, int n, const double* __restrict__ a, const double* __restrict__ b,
                                     const double* __restrict__ c, double* __restrict__ r, double* __restrict__ cc)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const long o = (long)s * n;
    double bb = b[o];
    cc[o] = c[o] / bb;
    r[o] = r[o] / bb;
    for (int i = 1; i < n; ++i) {
        bb = b[o + i] - cc[o + i - 1] * a[o + i];
        cc[o + i] = c[o + i] / bb;
        r[o + i] = (r[o + i] - r[o + i - 1] * a[o + i]) / bb;
    }
    for (int i = n - 2; i >= 0; --i) r[o + i] = r[o + i] - r[o + i + 1] * cc[o + i];
}

__global__ void k_divide(long n, double* __restrict__ x, double d)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) x[t] = x[t] / d;
}

}  // namespace

extern "C" int pllgpu_set_timestep(pllgpu_ctx* ctx, double ts)
{
    if (!ctx) return PLLGPU_EINVAL;
    ctx->timestep = ts;
    return set_scalar(ctx, S_TIMESTEP, ts);
}

extern "C" int pllgpu_set_tval(pllgpu_ctx* ctx, double t)
{
    if (!ctx) return PLLGPU_EINVAL;
    return set_scalar(ctx, S_TVAL, t);
}

extern "C" int pllgpu_acoef(pllgpu_ctx* ctx, int var, int which, double* abc9)
{
    if (!ctx || var < 0 || var > 3 || (which != 0 && which != 1) || !abc9) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    if (int e = materialize(ctx)) return e;
    const long ne = ctx->nelem;
    DevBuf buf;
    if (!buf.alloc(sizeof(double) * 9 * (size_t)ne)) return fail(ctx, PLLGPU_ECUDA);
    CK(cudaMemsetAsync(buf.p, 0, sizeof(double) * 9 * (size_t)ne, ctx->st));
    MuPtrs<double> m = which ? ctx->mu_new() : ctx->mu_old();
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

extern "C" int pllgpu_weno_batch(int n, const double* v5, double* out)
{
    if (n < 0 || !v5 || !out) return PLLGPU_EINVAL;
    if (n == 0) return PLLGPU_OK;
    DevBuf dv, dout;
    if (!dv.alloc(sizeof(double) * 5 * (size_t)n) || !dout.alloc(sizeof(double) * (size_t)n)) return PLLGPU_ECUDA;
    if (cudaMemcpy(dv.p, v5, sizeof(double) * 5 * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    k_weno_batch<<<(n + 127) / 128, 128>>>(n, dv.d(), dout.d());
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(out, dout.p, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return PLLGPU_ECUDA;
    return PLLGPU_OK;
}

extern "C" int pllgpu_tridiag_1rhs_batch(int N, int n, const double* a, const double* b, const double* c,
                                         double* r)
{
    if (N < 0 || n < 1 || !a || !b || !c || !r) return PLLGPU_EINVAL;
    if (N == 0) return PLLGPU_OK;
    const size_t bytes = sizeof(double) * (size_t)N * n;
    DevBuf da, db, dc, dr, dcc;
    if (!da.alloc(bytes) || !db.alloc(bytes) || !dc.alloc(bytes) || !dr.alloc(bytes) || !dcc.alloc(bytes))
        return PLLGPU_ECUDA;
    if (cudaMemcpy(da.p, a, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(db.p, b, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dc.p, c, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dr.p, r, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    k_tridiag_1rhs_batch<<<(N + 127) / 128, 128>>>(N, n, da.d(), db.d(), dc.d(), dr.d(), dcc.d());
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(r, dr.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return PLLGPU_ECUDA;
    return PLLGPU_OK;
}

extern "C" int pllgpu_idct2d_batch(int n0, int n1, int howmany, const double* in, double* out)
{
    if (n0 < 1 || n1 < 1 || howmany < 0 || !in || !out) return PLLGPU_EINVAL;
    if (howmany == 0) return PLLGPU_OK;
    const long per = (long)n0 * n1, tot = per * howmany;
    const size_t bytes = sizeof(double) * (size_t)tot;
    std::vector<double> T0((size_t)n0 * n0), T1((size_t)n1 * n1);
    dct_matrix(1, n0, T0.data());
    dct_matrix(1, n1, T1.data());
    DevBuf dT0, dT1, dx, dtmp, dy;
    if (!dT0.alloc(sizeof(double) * T0.size()) || !dT1.alloc(sizeof(double) * T1.size()) || !dx.alloc(bytes) ||
        !dtmp.alloc(bytes) || !dy.alloc(bytes))
        return PLLGPU_ECUDA;
    if (cudaMemcpy(dT0.p, T0.data(), sizeof(double) * T0.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dT1.p, T1.data(), sizeof(double) * T1.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dx.p, in, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return PLLGPU_ECUDA;
    GemmDesc d1{n0, n1, n1, howmany, per, n1, 1, 0, 1, n1, per, n1, 1, 0.0, 0};
    k_gemm_seq<double><<<dim3((n1 + 63) / 64, (n0 + 63) / 64, howmany), 256>>>(d1, dx.d(), dT1.d(), dtmp.d());
    GemmDesc d2{n0, n1, n0, howmany, 0, n0, 1, per, n1, 1, per, n1, 1, 0.0, 0};
    k_gemm_seq<double><<<dim3((n1 + 63) / 64, (n0 + 63) / 64, howmany), 256>>>(d2, dT0.d(), dtmp.d(), dy.d());
    // fftw_3d.h:101 divides by (double)(4*N)
    k_divide<<<(int)((tot + 255) / 256), 256>>>(tot, dy.d(), (double)(4 * per));
    if (cudaGetLastError() != cudaSuccess) return PLLGPU_ECUDA;
    if (cudaMemcpy(out, dy.p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return PLLGPU_ECUDA;
    return PLLGPU_OK;
}
