/*
 * pllcart3d_gpu.h - C ABI of the B200 implementation of pllcart3d's
 * RK3 / Crank-Nicolson time step (csdms-contrib/pllcart3d).
 *
 * Two layers, both plain C:
 *
 * 1. The device API (libpllgpu.so, prefix pllgpu_): a context that owns the
 *    solver state in HBM, runs whole time steps on the GPU (one CUDA graph
 *    per step) and runs each step routine of the reference on its own for
 *    per-routine parity.  Fields cross the boundary as contiguous float64
 *    arrays over the padded box (nx+6) x (ny+2) x (nz+2), z fastest - the
 *    element order of the reference's double***[i][j][k] arrays
 *    (allocate_3d_calloc.h:46-64).
 *
 * 2. The drop-in layer (libpllcart3d_dropin.so): the reference's own
 *    step-routine names and signatures (global_function_decl.h:7-26,36-42,
 *    pll_tridiag.c:152, fftw_3d.h:3-5) over its structures_3d.h types, so
 *    that pllcart3d.c links against it in place of its CPU routines.  Those
 *    prototypes take the reference's Grid/Velo/Conc/Visc/Tds types and are
 *    declared by the reference's own headers; they are listed at the end of
 *    this file with layout-identical mirror types (the reference names a
 *    member `new`, which is why the mirrors rename it).
 *
 * Errors: every pllgpu_ call returns PLLGPU_OK or an error code; the status
 * of a context is sticky until pllgpu_clear_status.  Nothing here traps or
 * exits the process; the reference's exit(1) paths (NaN in find_max,
 * pllcart3d.c:3568-3588; slope-parameter non-convergence, L813-818) become
 * PLLGPU_ENAN / PLLGPU_ENOCONV.
 */
#ifndef PLLCART3D_GPU_H
#define PLLCART3D_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PLLGPU_OK 0
#define PLLGPU_ENAN 1      /* NaN/Inf met in the CFL scan (find_max's guard)  */
#define PLLGPU_ECUDA 2     /* a CUDA call failed                               */
#define PLLGPU_ETIMEOUT 3  /* a bounded device wait gave up                    */
#define PLLGPU_EBOUNDS 4   /* a kernel self-check found a bad index            */
#define PLLGPU_EINVAL 5    /* bad argument (size, field id, routine id)        */
#define PLLGPU_ENOCONV 6   /* slope_parameter bisection did not converge       */

/* precision forms */
#define PLLGPU_FP64 0      /* plain: the reference's FP64 arithmetic           */
#define PLLGPU_MIXED 1     /* FP32 state, WENO/stress/ADI in FP32, split-TF32
                              tensor-core DCT, FP64 Poisson mode solve and
                              FP64 reductions                                  */
#define PLLGPU_MIXED64 2   /* FP64 state and FP64 arithmetic except the WENO5
                              nonlinear weights, evaluated in FP32 from the
                              FP64 divided differences                         */

/* run parameters: the values of param.input that the step reads
 * (input() pllcart3d.c:271-350); M = Vratio, Vnorm = 0 (L400-403) */
typedef struct pllgpu_params {
    int nx, ny, nz;        /* Nx_cell_global, Ny_cell_global, Nz_cell_global */
    int nmvp;              /* Nmvp: 0 mu = exp(M c), 1 non-monotonic law      */
    double X1, X2, Y1, Y2, Z1, Z2;
    double Re, Pe, Vratio, Fx, Fy, CFLmax, Timestep, Mum, Lambda;
    int precision;         /* PLLGPU_FP64, PLLGPU_MIXED or PLLGPU_MIXED64      */
    int exact_dct;         /* 1: DCT sums in sequential order (bitwise with
                              the CPU restatement; FP64: the reference's
                              operation order throughout), and in the precision form
                              every line / mode solve the sequential Thomas
                              sweep; 0: tensor-core DCT, and in the precision
                              form the partitioned line solves and, with the
                              tcgen05 DCT, the FP32-scratch mode solve        */
    int use_graph;         /* 1: replay each step as one CUDA graph            */
    int dct_kernel;        /* precision form, exact_dct 0: 0 = tcgen05 split-TF32
                              GEMMs (persistent, one CTA per SM) where ny, nz
                              are 128 or 256, else mma.sync; 1 = mma.sync
                              split-TF32 always; 2 = tcgen05, one tile per CTA */
    int explicit_kernel;   /* explicit operator, exact_dct 0: 0 = default (FP64
                              forms: TMA-staged plane-marching kernel; the
                              precision form: cell pairs in FP32x2), 1 = the
                              per-cell kernel (FP64) / cell pairs (FP32), 2 =
                              the TMA-staged kernel in either form           */
    int reserved[3];
} pllgpu_params;

typedef struct pllgpu_ctx pllgpu_ctx;

/* field ids (pllgpu_field_id maps the names "c_old" ... "div") */
enum {
    PLLGPU_C_OLD = 0, PLLGPU_C_NEW, PLLGPU_C_HN, PLLGPU_C_HNM1,
    PLLGPU_U_OLD, PLLGPU_U_NEW, PLLGPU_U_HN, PLLGPU_U_HNM1, PLLGPU_U_PG,
    PLLGPU_V_OLD, PLLGPU_V_NEW, PLLGPU_V_HN, PLLGPU_V_HNM1, PLLGPU_V_PG,
    PLLGPU_W_OLD, PLLGPU_W_NEW, PLLGPU_W_HN, PLLGPU_W_HNM1, PLLGPU_W_PG,
    PLLGPU_MU_OLD_CELL, PLLGPU_MU_OLD_XY, PLLGPU_MU_OLD_XZ, PLLGPU_MU_OLD_YZ,
    PLLGPU_MU_NEW_CELL, PLLGPU_MU_NEW_XY, PLLGPU_MU_NEW_XZ, PLLGPU_MU_NEW_YZ,
    PLLGPU_PHI, PLLGPU_DIV,
    PLLGPU_NFIELDS
};

/* routine ids for pllgpu_routine; scalars in[] as listed, out[0] result */
enum {
    PLLGPU_R_CONCENTRATION = 0,   /* concentration L555-719: dt,g,r,vbulk     */
    PLLGPU_R_VISCOSITY_NEW,       /* calculate_viscosity(c_new) L843-886      */
    PLLGPU_R_XMOM,                /* xmom L952-1107: dt,g,r,vbulk             */
    PLLGPU_R_YMOM,                /* ymom L1110-1260                          */
    PLLGPU_R_ZMOM,                /* zmom L1263-1408                          */
    PLLGPU_R_VELO_GHOSTS,         /* update_velo_boundary L2701-2755 /
                                     update_veloghost_points L2810-2885       */
    PLLGPU_R_DIVERGENCE,          /* divergence L1983-1999                    */
    PLLGPU_R_PHISOLVER,           /* phisolver_dct L2002-2130: dt,g,r         */
    PLLGPU_R_PHI_GHOSTS,          /* update_phi_ghosts L2758-2807             */
    PLLGPU_R_VELO_CORRECTION,     /* velo_correction L2133-2227: dt,g,r       */
    PLLGPU_R_PRESSURE_GRADIENT,   /* pressure_gradient L2964-3044: dt,g,r     */
    PLLGPU_R_ROTATE,              /* update_old_conc/velo/visc L3402-3452     */
    PLLGPU_R_BULK_VELO,           /* bulk_velo L3381-3398 -> out[0]           */
    PLLGPU_R_FIND_CFL,            /* find_cfl L3095-3118 -> out[0]            */
    PLLGPU_R_SUBSTEP,             /* one RK substep L164-194: dt, rk          */
    PLLGPU_R_VISCOSITY_EXP,       /* calculate_viscosity(c_new) L843-886,
                                     mu = exp(M c) whatever Nmvp is           */
    PLLGPU_R_VISCOSITY_NMVP,      /* calculate_viscosity_nmvp L889-948: cm    */
    PLLGPU_R_SLOPE_PARAMETER,     /* slope_parameter(c_new) L722-840 -> out[0]*/
    PLLGPU_NROUTINES
};

pllgpu_ctx *pllgpu_create(const pllgpu_params *p, int device);
void pllgpu_destroy(pllgpu_ctx *ctx);
int pllgpu_field_id(const char *name);
int pllgpu_dims(const pllgpu_ctx *ctx, int *dims6); /* NX NY NZ nx ny nz */
int pllgpu_set_field(pllgpu_ctx *ctx, int field, const double *host);
int pllgpu_get_field(pllgpu_ctx *ctx, int field, double *host);
/* device address and element strides (i, j) of a field in the current
 * roles; valid until the next step or rotate */
int pllgpu_device_field(pllgpu_ctx *ctx, int field, double **dptr,
                        long *stride_i, long *stride_j);
/* start-up after the initial *_new fields are set: pllcart3d.c:81-83
 * (ghost fill, new -> old), 126-148 (viscosity of c_old, slope parameter)
 * and 150-154 (diffusive cap of Timestep) */
int pllgpu_start(pllgpu_ctx *ctx);
/* start-up after pllgpu_read_restart (pllcart3d.c:111 then 126-154): the
 * viscosity of c_old (and the slope parameter, which the reference computes
 * from c->new), no ghost fill, no new -> old copy; tval as read */
int pllgpu_resume(pllgpu_ctx *ctx, double tval);
/* n full time steps, pllcart3d.c:158-195, dt from the device CFL scan */
int pllgpu_steps(pllgpu_ctx *ctx, int nsteps);
/* n steps, copying the four initial fields in from host and c,u,v,w out to
 * host inside the call (end-to-end entry point) */
int pllgpu_run_host(pllgpu_ctx *ctx, int nsteps, const double *c0,
                    const double *u0, const double *v0, const double *w0,
                    double *c, double *u, double *v, double *w);
int pllgpu_routine(pllgpu_ctx *ctx, int routine, const double *in, double *out);
int pllgpu_sync(pllgpu_ctx *ctx);
int pllgpu_status(const pllgpu_ctx *ctx);
void pllgpu_clear_status(pllgpu_ctx *ctx);
double pllgpu_last_dt(pllgpu_ctx *ctx);
double pllgpu_timestep(const pllgpu_ctx *ctx);
double pllgpu_tval(pllgpu_ctx *ctx);
const char *pllgpu_error_string(int code);
/* number of kernel launches one time step issues */
int pllgpu_kernels_per_step(const pllgpu_ctx *ctx);
/* the CUDA stream (cudaStream_t) every kernel of the context runs on */
void *pllgpu_stream(pllgpu_ctx *ctx);
/* nsteps steps launched one kernel at a time with a CUDA event after each
 * launch: per kernel label (names: maxk slots of 32 chars) the summed
 * device time in ms and the number of launches; *nk = labels filled */
int pllgpu_profile_steps(pllgpu_ctx *ctx, int nsteps, int maxk, char *names,
                         double *total_ms, int *launches, int *nk);

/* FP64 diagnostics of the current state: out4[0] mass = sum c dV,
 * out4[1] max |div u|, out4[2] the L2 norm of div u, out4[3] the mixing
 * length = dx * #{x-planes with 0.01 < yz-mean of c < 0.99} (the yz mean
 * of conc_average, pllcart3d.c:3692-3704) */
int pllgpu_diagnostics(pllgpu_ctx *ctx, double *out4);
/* Timestep after the diffusive cap (pllcart3d.c:150-154) and the simulated
 * time, for hosts that run their own start-up */
int pllgpu_set_timestep(pllgpu_ctx *ctx, double timestep);
int pllgpu_set_tval(pllgpu_ctx *ctx, double tval);
/* implicit-operator coefficients of variable var (0 c, 1 u, 2 v, 3 w) from
 * the mu_old (which=0) or mu_new (which=1) arrays, A_conc/A_umom/A_vmom/
 * A_wmom (pllcart3d.c:1411-1536): abc9 holds 9 padded fields (a,b,c of x,
 * then y, then z), filled on the variable's unknown range, 0 elsewhere */
int pllgpu_acoef(pllgpu_ctx *ctx, int var, int which, double *abc9);

/* calculate_weno (pllcart3d.c:3455-3507) for n points: v5 holds the five
 * divided differences d1[kk + sign*m], m = 0..4, of each point */
int pllgpu_weno_batch(int n, const double *v5, double *out);
/* tridiag_1rhs (pllcart3d.c:3511-3536) for N systems of length n, host
 * buffers as pllgpu_tridiag_batch; a, b, c are left untouched */
int pllgpu_tridiag_1rhs_batch(int N, int n, const double *a, const double *b,
                              const double *c, double *r);
/* idct_3d's transform (fftw_3d.h:77-106): REDFT01 in both dimensions
 * followed by the division by 4*n0*n1 */
int pllgpu_idct2d_batch(int n0, int n1, int howmany, const double *in,
                        double *out);

/*
 * Batched line solve of pll_tridiag (pll_tridiag.c:152-158) on one rank:
 * N independent systems of length n, a/b/c/r each N*n contiguous host
 * doubles (system s at offset s*n); on return r holds the solution and b, c
 * the eliminated coefficients, as the reference leaves them.
 */
int pllgpu_tridiag_batch(int N, int n, const double *a, double *b, double *c,
                         double *r);

/*
 * Batched 2-d DCT of fftw_3d.h:45-106: `howmany` row-major n0 x n1 arrays
 * (n1 fastest), kind 0 = REDFT10 (DCT-II), 1 = REDFT01 (DCT-III), both
 * unnormalised as FFTW defines them.  Host buffers.
 */
int pllgpu_dct2d_batch(int kind, int n0, int n1, int howmany, const double *in,
                       double *out);

/* ---- snapshot, restart and diagnostic files ---------------------------- *
 * The reference's output routines on the resident state, writing its file
 * formats into `dir` (NULL: the working directory).  The device packs each
 * file's values, one copy brings them to pinned host memory.
 *   pllgpu_write_snapshot  write_to_file (pllcart3d.c:3047): caf%04dR000.bin,
 *                          float32 u,v,w (cell centres), c per interior cell;
 *                          only even (i,j,k) cells above 2e7 cells
 *   pllgpu_write_snapshot_ex  the same with the MPI rank of the file name and
 *                          subsample -1 (the reference's rule), 0 (all cells)
 *                          or 1 (even cells)
 *   pllgpu_write_restart   midfield (L3121): middata + midfield000.bin
 *   pllgpu_read_restart    intermediate (L3181): reads them into the 14
 *                          fields; follow with pllgpu_resume
 *   pllgpu_conc_average    conc_average (L3635): appends cavgy.bin,
 *                          cavgz.bin, cavgyz.bin
 *   pllgpu_find_wmax       find_wmax (L3606): appends (wmax, tval) to
 *                          wmax.bin when dir is given; wmax to *wmax_out
 *   pllgpu_find_max        find_max (L3539): appends the max |u|,|v|,|w|,|c|
 *                          block to Outscreen; maxval[4] / maxloc[12] out;
 *                          a NaN in c (old, new, explicit) writes the
 *                          reference's "nan in" line and returns PLLGPU_ENAN
 *                          where the reference calls exit(1)
 */
int pllgpu_write_snapshot(pllgpu_ctx *ctx, int fileno, const char *dir);
int pllgpu_write_snapshot_ex(pllgpu_ctx *ctx, int fileno, int rank,
                             const char *dir, int subsample);
int pllgpu_write_restart(pllgpu_ctx *ctx, int tstep, int fileno, double tval,
                         double outtime, double outmid, double cavgtime,
                         const char *dir);
int pllgpu_read_restart(pllgpu_ctx *ctx, const char *dir, int *tstep,
                        int *fileno, double *tval, double *outtime);
int pllgpu_conc_average(pllgpu_ctx *ctx, double tval, const char *dir);
int pllgpu_find_wmax(pllgpu_ctx *ctx, double tval, const char *dir,
                     double *wmax_out);
int pllgpu_find_max(pllgpu_ctx *ctx, const char *dir, double *maxval,
                    int *maxloc);

/* shift_conc (pllcart3d.c:3231, spline L3280): the spanwise wave
 * perturbation of c_old, each x line re-sampled at x - meshdx(z) by a natural
 * cubic spline; meshdx = ampli cos(2 pi z / lamb) (+ the sub-harmonic term
 * when subharm = 1).  The reference's Ampli, Lamb and Subharm of
 * param.input; it calls this once, at tval >= 2 with Wavpert = 1 (L247). */
int pllgpu_shift_conc(pllgpu_ctx *ctx, double ampli, double lamb, int subharm);

/* ---- launch-shape autotuner ----------------------------------------------
 * Times every launch-shape variant of the explicit operators (4) and the x/y
 * line solves (3) on `trial_steps` steps each (plus one warm-up step) and
 * keeps the fastest.  All variants compute bit-identical results, so the
 * trial steps are steps of the run; *steps_done reports how many. */
int pllgpu_autotune(pllgpu_ctx *ctx, int trial_steps, int *steps_done);
int pllgpu_tuning(pllgpu_ctx *ctx, int *explicit_variant, int *line_variant);
int pllgpu_set_tuning(pllgpu_ctx *ctx, int explicit_variant, int line_variant);

/* ---- ensembles ------------------------------------------------------------
 * n independent runs (each its own grid and parameters, params[i]) on one
 * device, advanced together by one CUDA graph launch per step.  Members
 * whose steps issue the same launches (the same grid and form) form a
 * class; the graph holds one branch per class and, by default, one launch
 * per stage for the whole class (each member reading its own arguments from
 * a device table).  Members are ordinary contexts (pllgpu_ensemble_member):
 * set their fields and read them with the calls above.  Every member
 * computes exactly what it computes alone.  No reference counterpart. */
typedef struct pllgpu_ensemble pllgpu_ensemble;
pllgpu_ensemble *pllgpu_ensemble_create(int n, const pllgpu_params *params,
                                        int device);
void pllgpu_ensemble_destroy(pllgpu_ensemble *ens);
int pllgpu_ensemble_size(const pllgpu_ensemble *ens);
pllgpu_ctx *pllgpu_ensemble_member(pllgpu_ensemble *ens, int i);
int pllgpu_ensemble_start(pllgpu_ensemble *ens);
int pllgpu_ensemble_steps(pllgpu_ensemble *ens, int nsteps);
int pllgpu_ensemble_autotune(pllgpu_ensemble *ens, int trial_steps,
                             int *steps_done);
int pllgpu_ensemble_launches_per_step(const pllgpu_ensemble *ens);
/* mode 1 (the default): one launch per stage and class; k >= 2: classes
 * split into groups of at most k members, one launch per stage and group;
 * 0: every member's own launches as its own branch.  Returns the previous
 * mode (negative: invalid arguments); the graphs are rebuilt on the next
 * steps call. */
int pllgpu_ensemble_set_batching(pllgpu_ensemble *ens, int mode);
/* branches (classes, or groups of a class) of the graphs last built (0
 * before the first steps call) */
int pllgpu_ensemble_classes(const pllgpu_ensemble *ens);

/* the whole state of src (fields of both buffer roles, viscosity,
 * pressure gradient, phi, device scalars) into dst, device to device; both
 * of the same grid and form.  No reference counterpart. */
int pllgpu_copy_state(pllgpu_ctx *dst, pllgpu_ctx *src);

/* cell-centred (u, v, w, c) float32 of every interior cell, i-j-k order
 * ([nx][ny][nz][4]), into / out of a caller's device buffer (16-byte
 * aligned): the state exchange of a learned model.  unpack writes c's
 * interior (with its y/z Neumann ghosts) and the interior faces of u, v, w
 * (mean of the two adjacent centres) into the *_new fields; boundary faces
 * keep their values.  No reference counterpart. */
int pllgpu_pack_cells(pllgpu_ctx *ctx, float *d_cells);
int pllgpu_unpack_cells(pllgpu_ctx *ctx, const float *d_cells);

/*
 * pllgpu_dct2d_batch without device allocation.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory
 * themselves or through this library (a host whose pool allocator owns the
 * device's memory; a caller that cannot accept the device synchronisation
 * that cudaMalloc/cudaFree may cause).  d_in and d_out are the caller's
 * device buffers (howmany*n0*n1 doubles each, as pllgpu_dct2d_batch lays
 * them out); the work runs on `stream` (a cudaStream_t, NULL for the legacy
 * default stream) and is not synchronised.  The two cosine matrices and the
 * intermediate array live in one fixed scratch array inside the library of
 * PLLGPU_DCT_NOALLOC_MAX_DOUBLES doubles (16 MiB) per device, held until the
 * process exits: n0*n0 + n1*n1 + howmany*n0*n1 must not exceed it
 * (PLLGPU_EINVAL and a message otherwise, checked without overflow before
 * any device work).  Any howmany that fits runs (the batch is launched in
 * chunks of at most 65535 arrays).  The first call on a device looks the
 * scratch address up on that device (make it current first).  Calls share
 * the scratch and it keeps the last call's contents, so calls that overlap
 * on the GPU (other streams, other threads) race; each call overwrites what
 * it reads, so none needs it cleared.  PLLGPU_ECUDA reports a failed launch
 * of this call's own kernels; an error left pending by earlier, unrelated
 * work is neither reported nor cleared.
 */
#define PLLGPU_DCT_NOALLOC_MAX_DOUBLES (1L << 21)
int pllgpu_dct2d_batch_noalloc(int kind, int n0, int n1, int howmany,
                               const double *d_in, double *d_out,
                               void *stream);

#ifdef __cplusplus
}
#endif

/* ------------------------------------------------------------------------ */
/* Drop-in layer (libpllcart3d_dropin.so).                                   */
/* The reference's own prototypes, over its structures_3d.h types, are:      */
/*   void concentration(double,double,double,double,Grid*,double***,        */
/*                      double***,double***,Conc*);          pllcart3d.c:555 */
/*   void calculate_viscosity(Grid*,double***,Visc*);         pllcart3d.c:843 */
/*   void calculate_viscosity_nmvp(Grid*,double***,Visc*,double);       L889 */
/*   double slope_parameter(Grid*,double***);                           L722 */
/*   void xmom(double,double,double,double,Grid*,Visc*,Visc*,double***,     */
/*             double***,double***,Velo*);                               L952 */
/*   void ymom(...same as xmom...);                                    L1110 */
/*   void zmom(double,double,double,double,Grid*,Visc*,Visc*,double***,     */
/*             double***,Velo*);                                        L1263 */
/*   void A_conc(Grid*,Conc*);  void A_umom(Grid*,Visc*,Velo*);       L1411 */
/*   void A_vmom(Grid*,Visc*,Velo*); void A_wmom(Grid*,Visc*,Velo*);  L1475 */
/*   void divergence(Grid*,double***,double***,double***,double***);  L1983 */
/*   void phisolver_dct(double,double,double,Grid*,double***,double***);    */
/*                                                                  L2002 */
/*   void velo_correction(double,double,double,Grid*,double***,Velo*,       */
/*                        Velo*,Velo*);                                L2133 */
/*   void update_velo_boundary(Grid*,Velo*,Velo*,Velo*);              L2701 */
/*   void update_phi_ghosts(Grid*,double***);                         L2758 */
/*   void update_veloghost_points(Grid*,Velo*,Velo*,Velo*);           L2810 */
/*   void pressure_gradient(double,double,double,Grid*,double***,Velo*,     */
/*                          Velo*,Velo*);                              L2964 */
/*   double find_cfl(Grid*,double***,double***,double***);            L3095 */
/*   double bulk_velo(Grid*,double***);                               L3381 */
/*   void update_old_conc(Conc*); void update_old_velo(Velo*,Velo*,Velo*);  */
/*   void update_old_visc(Visc*,Visc*);                          L3402-3452 */
/*   double calculate_weno(double*,int,int);                          L3455 */
/*   int tridiag_1rhs(int,double*,double*,double*,double*);           L3511 */
/*   void pll_tridiag(Tds*,int,int);                     pll_tridiag.c:152 */
/*   void plan_dct_3d(int,int,int); void fdct_3d(int,int,int,double***,     */
/*        double***); void idct_3d(int,int,int,double***,double***);        */
/*                                                            fftw_3d.h:3-5 */
/* plus the resident-state fast path:                                       */
/*   int  pllgpu_attach(Grid*,Velo*u,Velo*v,Velo*w,Conc*,Visc*mu_old,       */
/*                      Visc*mu_new,double***phi);                           */
/*   int  pllgpu_advance(int nsteps,double *tval);                          */
/*   int  pllgpu_sync_to_host(void);                                        */
/*   int  pllgpu_dropin_status(void); void pllgpu_finalize(void);           */
/*   pllgpu_ctx *pllgpu_dropin_context(void);  the context behind attach,   */
/*        for the resident snapshot / restart / diagnostic calls above      */
/* Layout-identical mirrors of the reference types follow.                   */
/* ------------------------------------------------------------------------ */
typedef struct pll_tds {          /* Tds, structures_3d.h:2-8 */
    double *acof, *bcof, *ccof, *rhs;
} pll_tds;
typedef struct pll_tri_abc {      /* Tri_abc, structures_3d.h:11-16 */
    double a, b, c;
} pll_tri_abc;
typedef struct pll_velo {         /* Velo, structures_3d.h:19-27 */
    int nx_max, ny_max, nz_max;
    int istart, iend, jstart, jend, kstart, kend;
    double ***next, ***old;       /* `new`, `old` */
    double ***pg;
    double ***explicit_n, ***explicit_nm1;
    pll_tri_abc ***Ax, ***Ay, ***Az;
} pll_velo;
typedef struct pll_conc {         /* Conc, structures_3d.h:30-37 */
    int nx_max, ny_max, nz_max;
    int istart, iend, jstart, jend, kstart, kend;
    double ***next, ***old;
    double ***explicit_n, ***explicit_nm1;
    pll_tri_abc ***Ax, ***Ay, ***Az;
} pll_conc;
typedef struct pll_visc {         /* Visc, structures_3d.h:40-48 */
    int nx_max, ny_max, nz_max;
    double ***cell, ***xy, ***xz, ***yz;
} pll_visc;
typedef struct pll_grid {         /* Grid, structures_3d.h:50-60 */
    int istart, iend, jstart, jend, kstart, kend;
    int nx_cell, ny_cell, nz_cell;
    int nx_max, ny_max, nz_max;
    int nmax_xyz, nx_global_offset;
    double dx, dy, dz;
    double *X, *Y, *Z;
    double *Xc, *Yc, *Zc;
} pll_grid;

#endif
