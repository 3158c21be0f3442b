// Device context of the pllcart3d B200 step: the state buffers of both
// precision forms and the bookkeeping shared by the orchestration units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/pllcart3d_gpu.h"
#include "aux_kernels.cuh"
#include "batch.cuh"
#include "common.cuh"
#include "dct_kernels.cuh"
#include "host_util.h"
#include "step_kernels.cuh"


namespace pll {

template <typename real>
struct Bufs {
    real* q[4][2] = {};     // c, u, v, w : [buffer]
    real* H[4][2] = {};
    real* mu[2][4] = {};    // [buffer][cell, xy, xz, yz]
    real* pg[4] = {};       // u, v, w at 1..3
    real* phi = nullptr;
    real* div = nullptr;
    real* S = nullptr;      // ADI right-hand side / eliminated rhs
    real* cc = nullptr;     // Thomas scratch
    real* dct1 = nullptr;   // compact nx*ny*nz Poisson buffers
    real* dct2 = nullptr;
    real *Ty = nullptr, *Tz = nullptr, *Tiy = nullptr, *Tiz = nullptr;
};

// tcgen05 DCT passes of the precision form: tensor maps of the four passes
// (A = the data, Bh / Bl = the cosine matrix's TF32 head and tail)
struct UmmaPlan {
    bool on = false;
    int sms = 148;   // persistent grid: one CTA per SM
    CUtensorMap a[4], bh[4], bl[4];
    float* Thi[4] = {};
    float* Tlo[4] = {};
};

}  // namespace pll

using namespace pll;

struct pllgpu_ctx {
    pllgpu_params P;
    Geo G;
    Rng Rg, Rv[4];
    Consts K;
    int dev = 0;
    bool mixed = false;
    cudaStream_t st = nullptr;
    long nelem = 0;             // elements of one padded field
    Bufs<double> b64;           // state of the FP64 form
    Bufs<float> b32;            // state of the mixed form
    double *mode_cc = nullptr, *mode_rr = nullptr;  // FP64 Poisson mode scratch
    double* stage64 = nullptr;  // one padded FP64 field (mixed-form transfers)
    double *lam_y = nullptr, *lam_z = nullptr;
    // FP64 form's FFT DCT passes (power-of-two planes): per axis (0 y, 1 z)
    // cos / sin of 2 pi m / N and of pi k / (2N)
    bool fft_on = false;
    bool xt_on = false;         // FP64 form: TMA-staged marching explicit operator
    double2 *fft_tw[2] = {nullptr, nullptr}, *fft_wq[2] = {nullptr, nullptr};
    UmmaPlan um;                // precision form's tensor-core DCT (when shapes allow)
    double* scal = nullptr;     // device scalars (S_*)
    int* status = nullptr;      // device sticky status bits
    double* work = nullptr;     // slope-parameter scratch
    double* red = nullptr;      // multi-block reduction partials (RED_DOUBLES)
    unsigned* ticket = nullptr; // last-block tickets of those reductions (2, self-resetting)
    double* diag = nullptr;     // per-plane diagnostics + results
    int cur = 0;                // buffer index holding the "old" role
    bool resync_c = false;      // after a restart: copy c's buffers once (resume)
    int tune_exp = 0;           // launch-shape variants (autotuner): explicit-
    int tune_line = 1;          // operator block, x/y line-solve block
    bool rotated = false;       // fast steps ran: "new" roles are stale and
                                // logically equal to "old" (see materialize)
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    bool graphs_ready = false;
    double timestep = 0;
    int err = PLLGPU_OK;
    int launches_per_step = 0;
    int counting = 0;
    bool profiling = false;
    std::vector<pll::LaunchRec*>* rec = nullptr;   // recording: launches are stored, not issued
    std::vector<cudaEvent_t> ev_pool;
    std::vector<const char*> ev_label;
    std::vector<void*> allocs;
};

namespace pll {

template <typename real> Bufs<real>& bufs(pllgpu_ctx* c);
template <> inline Bufs<double>& bufs<double>(pllgpu_ctx* c) { return c->b64; }
template <> inline Bufs<float>& bufs<float>(pllgpu_ctx* c) { return c->b32; }

template <typename real> real* q_old(pllgpu_ctx* c, int v) { return bufs<real>(c).q[v][c->cur]; }
template <typename real> real* q_new(pllgpu_ctx* c, int v) { return bufs<real>(c).q[v][1 - c->cur]; }
template <typename real> real* h_n(pllgpu_ctx* c, int v) { return bufs<real>(c).H[v][1 - c->cur]; }
template <typename real> real* h_nm1(pllgpu_ctx* c, int v) { return bufs<real>(c).H[v][c->cur]; }
template <typename real> MuPtrs<real> mu_old(pllgpu_ctx* c)
{
    Bufs<real>& B = bufs<real>(c);
    return {B.mu[c->cur][0], B.mu[c->cur][1], B.mu[c->cur][2], B.mu[c->cur][3]};
}
template <typename real> MuPtrs<real> mu_new(pllgpu_ctx* c)
{
    Bufs<real>& B = bufs<real>(c);
    return {B.mu[1 - c->cur][0], B.mu[1 - c->cur][1], B.mu[1 - c->cur][2], B.mu[1 - c->cur][3]};
}

}  // namespace pll
