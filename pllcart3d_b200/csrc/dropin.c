/*
 * Drop-in layer: the reference's step routines under their own names and
 * signatures (global_function_decl.h:7-26,36-42; pll_tridiag.c:152;
 * fftw_3d.h:3-5), over its structures_3d.h types, executed on the GPU
 * through the pllgpu_ device API.  Linking pllcart3d.c against this library
 * instead of its own definitions of these routines moves every stage of the
 * time step (pllcart3d.c:158-195) onto the GPU with the host loop
 * unchanged.
 *
 * Per-routine calls keep the reference's ownership: the caller owns every
 * double*** array; a call uploads the arrays the routine reads, runs the
 * routine on the device and writes back the arrays it writes, row by row
 * (rows are separately calloc'ed, allocate_3d_calloc.h:58).  The resident
 * fast path (pllgpu_attach / pllgpu_advance / pllgpu_sync_to_host) keeps the
 * state in HBM across many steps instead.
 *
 * Compiled as C because structures_3d.h names a member `new`; the mirror
 * types of pllcart3d_gpu.h have the same layout.
 *
 * The reference's run parameters are its globals (global_variables.h): the
 * weak definitions below make the library loadable on its own; the
 * definitions in pllcart3d.c take precedence when it is linked in.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pllcart3d_gpu.h"

typedef pll_grid Grid;
typedef pll_velo Velo;
typedef pll_conc Conc;
typedef pll_visc Visc;
typedef pll_tds Tds;
typedef pll_tri_abc Tri_abc;

/* reference globals (global_variables.h:2-18) */
__attribute__((weak)) int Nx_cell_global, Ny_cell_global, Nz_cell_global;
__attribute__((weak)) int Nx_ghost, Ny_ghost, Nz_ghost;
__attribute__((weak)) int Nmvp;
__attribute__((weak)) double X1, X2, Y1, Y2, Z1, Z2;
__attribute__((weak)) double Re, Pe, Vratio, Fx, Fy, CFLmax, Timestep;
__attribute__((weak)) double M, Vnorm, Mum, Lambda;

static pllgpu_ctx *g_ctx;
static pllgpu_params g_p;
static double *g_stage;        /* one padded field, contiguous */
static double *g_abc;          /* 9 padded fields of coefficients */
static int g_status;
static const Visc *g_asrc[4];  /* viscosity each variable's A was built from */
/* plan_dct_3d dimensions */
static int g_dct_n1, g_dct_n2, g_dct_nt;
/* resident fast path */
static Grid *a_grid;
static Velo *a_u, *a_v, *a_w;
static Conc *a_c;
static Visc *a_mu_old, *a_mu_new;
static double ***a_phi;

static int record(int code)
{
    if (code != PLLGPU_OK && g_status == PLLGPU_OK) {
        g_status = code;
        fprintf(stderr, "pllcart3d drop-in: %s\n", pllgpu_error_string(code));
    }
    return code;
}

int pllgpu_dropin_status(void) { return g_status; }

/* context for the grid of this run (re-created when the size changes) */
static pllgpu_ctx *ctx_for(const Grid *g)
{
    if (g_ctx && g_p.nx == g->nx_cell && g_p.ny == g->ny_cell && g_p.nz == g->nz_cell)
        return g_ctx;
    if (g_ctx) pllgpu_destroy(g_ctx);
    free(g_stage);
    free(g_abc);
    g_abc = NULL;
    memset(&g_p, 0, sizeof(g_p));
    g_p.nx = g->nx_cell;
    g_p.ny = g->ny_cell;
    g_p.nz = g->nz_cell;
    g_p.nmvp = Nmvp;
    g_p.X1 = X1; g_p.X2 = X2; g_p.Y1 = Y1; g_p.Y2 = Y2; g_p.Z1 = Z1; g_p.Z2 = Z2;
    g_p.Re = Re; g_p.Pe = Pe;
    g_p.Vratio = M; /* the step reads M (= Vratio, pllcart3d.c:400) */
    g_p.Fx = Fx; g_p.Fy = Fy; g_p.CFLmax = CFLmax; g_p.Timestep = Timestep;
    g_p.Mum = Mum; g_p.Lambda = Lambda;
    g_p.precision = PLLGPU_FP64;
    g_p.exact_dct = 0;
    g_p.use_graph = 1;
    g_ctx = pllgpu_create(&g_p, 0);
    if (!g_ctx) {
        record(PLLGPU_ECUDA);
        return NULL;
    }
    g_stage = (double *)malloc(sizeof(double) * (size_t)g->nx_max * g->ny_max * g->nz_max);
    return g_ctx;
}

/* row-by-row gather / scatter of a double*** field */
static void gather(const Grid *g, double ***f, double *dst)
{
    int i, j;
    for (i = 0; i < g->nx_max; i++)
        for (j = 0; j < g->ny_max; j++)
            memcpy(dst + ((long)i * g->ny_max + j) * g->nz_max, f[i][j], sizeof(double) * g->nz_max);
}

static void scatter(const Grid *g, const double *src, double ***f)
{
    int i, j;
    for (i = 0; i < g->nx_max; i++)
        for (j = 0; j < g->ny_max; j++)
            memcpy(f[i][j], src + ((long)i * g->ny_max + j) * g->nz_max, sizeof(double) * g->nz_max);
}

static int up(const Grid *g, int field, double ***f)
{
    if (!f) return PLLGPU_OK;
    gather(g, f, g_stage);
    return record(pllgpu_set_field(g_ctx, field, g_stage));
}

static int down(const Grid *g, int field, double ***f)
{
    int e;
    if (!f) return PLLGPU_OK;
    e = pllgpu_get_field(g_ctx, field, g_stage);
    if (e == PLLGPU_OK) scatter(g, g_stage, f);
    return record(e);
}

static int up_visc(const Grid *g, int first, const Visc *mu)
{
    int e = 0;
    e = e || up(g, first + 0, mu->cell);
    e = e || up(g, first + 1, mu->xy);
    e = e || up(g, first + 2, mu->xz);
    e = e || up(g, first + 3, mu->yz);
    return e ? g_status : PLLGPU_OK;
}

static int down_visc(const Grid *g, int first, Visc *mu)
{
    int e = 0;
    e = e || down(g, first + 0, mu->cell);
    e = e || down(g, first + 1, mu->xy);
    e = e || down(g, first + 2, mu->xz);
    e = e || down(g, first + 3, mu->yz);
    return e ? g_status : PLLGPU_OK;
}

static int run(int routine, double a, double b, double c, double d, double *out)
{
    double in[4];
    in[0] = a; in[1] = b; in[2] = c; in[3] = d;
    return record(pllgpu_routine(g_ctx, routine, in, out));
}

/* coefficient triples of variable var from the mu_new slot into the
 * reference's Tri_abc arrays, on the variable's unknown range only (the
 * rest of a Tri_abc row is never initialised by the reference,
 * allocate_3d_calloc.h:97) */
static void fill_abc(const Grid *g, int var, int is, int ie, int js, int je, int ks, int ke,
                     Tri_abc ***Ax, Tri_abc ***Ay, Tri_abc ***Az)
{
    long ne = (long)g->nx_max * g->ny_max * g->nz_max;
    int i, j, k, ax;
    Tri_abc ***A[3];
    if (!g_abc) g_abc = (double *)malloc(sizeof(double) * 9 * (size_t)ne);
    if (record(pllgpu_acoef(g_ctx, var, 1, g_abc))) return;
    A[0] = Ax; A[1] = Ay; A[2] = Az;
    for (ax = 0; ax < 3; ax++)
        for (i = is; i <= ie; i++)
            for (j = js; j <= je; j++)
                for (k = ks; k <= ke; k++) {
                    long id = ((long)i * g->ny_max + j) * g->nz_max + k;
                    A[ax][i][j][k].a = g_abc[(3 * ax + 0) * ne + id];
                    A[ax][i][j][k].b = g_abc[(3 * ax + 1) * ne + id];
                    A[ax][i][j][k].c = g_abc[(3 * ax + 2) * ne + id];
                }
}

/* ---- step routines ------------------------------------------------------ */

/* concentration, pllcart3d.c:555-719 */
void concentration(double dt, double g, double r, double vbulk, Grid *grid, double ***un,
                   double ***vn, double ***wn, Conc *c)
{
    if (!ctx_for(grid)) return;
    if (up(grid, PLLGPU_C_OLD, c->old) || up(grid, PLLGPU_C_NEW, c->next) ||
        up(grid, PLLGPU_C_HN, c->explicit_n) || up(grid, PLLGPU_C_HNM1, c->explicit_nm1) ||
        up(grid, PLLGPU_U_NEW, un) || up(grid, PLLGPU_V_NEW, vn) || up(grid, PLLGPU_W_NEW, wn))
        return;
    if (run(PLLGPU_R_CONCENTRATION, dt, g, r, vbulk, NULL)) return;
    down(grid, PLLGPU_C_NEW, c->next);
    down(grid, PLLGPU_C_HN, c->explicit_n);
}

/* calculate_viscosity, pllcart3d.c:843-886 */
void calculate_viscosity(Grid *grid, double ***cn, Visc *mu)
{
    if (!ctx_for(grid)) return;
    if (up(grid, PLLGPU_C_NEW, cn) || up_visc(grid, PLLGPU_MU_NEW_CELL, mu)) return;
    if (run(PLLGPU_R_VISCOSITY_EXP, 0, 0, 0, 0, NULL)) return;
    down_visc(grid, PLLGPU_MU_NEW_CELL, mu);
}

/* calculate_viscosity_nmvp, pllcart3d.c:889-948 */
void calculate_viscosity_nmvp(Grid *grid, double ***cn, Visc *mu, double cm)
{
    if (!ctx_for(grid)) return;
    if (up(grid, PLLGPU_C_NEW, cn) || up_visc(grid, PLLGPU_MU_NEW_CELL, mu)) return;
    if (run(PLLGPU_R_VISCOSITY_NMVP, cm, 0, 0, 0, NULL)) return;
    down_visc(grid, PLLGPU_MU_NEW_CELL, mu);
}

/* slope_parameter, pllcart3d.c:722-840 (one rank) */
double slope_parameter(Grid *grid, double ***cn)
{
    double cm = 0.0;
    if (!ctx_for(grid)) return cm;
    if (up(grid, PLLGPU_C_NEW, cn)) return cm;
    run(PLLGPU_R_SLOPE_PARAMETER, 0, 0, 0, 0, &cm);
    return cm;
}

/* A_conc / A_umom / A_vmom / A_wmom, pllcart3d.c:1411-1536 */
void A_conc(Grid *grid, Conc *c)
{
    if (!ctx_for(grid)) return;
    fill_abc(grid, 0, c->istart, c->iend, c->jstart, c->jend, c->kstart, c->kend, c->Ax, c->Ay, c->Az);
}

static void a_mom(Grid *grid, int var, Visc *mu, Velo *q)
{
    if (!ctx_for(grid)) return;
    if (up_visc(grid, PLLGPU_MU_NEW_CELL, mu)) return;
    fill_abc(grid, var, q->istart, q->iend, q->jstart, q->jend, q->kstart, q->kend, q->Ax, q->Ay, q->Az);
    g_asrc[var] = mu;
}

void A_umom(Grid *grid, Visc *mu, Velo *u) { a_mom(grid, 1, mu, u); }
void A_vmom(Grid *grid, Visc *mu, Velo *v) { a_mom(grid, 2, mu, v); }
void A_wmom(Grid *grid, Visc *mu, Velo *w) { a_mom(grid, 3, mu, w); }

/* xmom / ymom / zmom, pllcart3d.c:952-1408: the explicit part uses mu_old
 * (the viscosity the stored A was built from), the implicit part rebuilds A
 * from mu_new and leaves it in the Tri_abc arrays (L991, L1148, L1300) */
static void momentum(int var, double dt, double g, double r, double vb, Grid *grid, Visc *mu_old,
                     Visc *mu_new, double ***cn, double ***uo, double ***vo, double ***wo, Velo *q)
{
    static const int first[4] = {0, PLLGPU_U_OLD, PLLGPU_V_OLD, PLLGPU_W_OLD};
    static const int routine[4] = {0, PLLGPU_R_XMOM, PLLGPU_R_YMOM, PLLGPU_R_ZMOM};
    int f = first[var];
    if (!ctx_for(grid)) return;
    if (up(grid, f + 0, q->old) || up(grid, f + 1, q->next) || up(grid, f + 2, q->explicit_n) ||
        up(grid, f + 3, q->explicit_nm1) || up(grid, f + 4, q->pg) ||
        up_visc(grid, PLLGPU_MU_OLD_CELL, mu_old) || up_visc(grid, PLLGPU_MU_NEW_CELL, mu_new) ||
        (cn && up(grid, PLLGPU_C_NEW, cn)))
        return;
    if (var != 1 && up(grid, PLLGPU_U_OLD, uo)) return;
    if (var != 2 && up(grid, PLLGPU_V_OLD, vo)) return;
    if (var != 3 && up(grid, PLLGPU_W_OLD, wo)) return;
    if (run(routine[var], dt, g, r, vb, NULL)) return;
    if (down(grid, f + 1, q->next) || down(grid, f + 2, q->explicit_n)) return;
    fill_abc(grid, var, q->istart, q->iend, q->jstart, q->jend, q->kstart, q->kend, q->Ax, q->Ay, q->Az);
    g_asrc[var] = mu_new;
}

void xmom(double dt, double g, double r, double vb, Grid *grid, Visc *mu_old, Visc *mu_new,
          double ***cn, double ***vold, double ***wold, Velo *u)
{
    momentum(1, dt, g, r, vb, grid, mu_old, mu_new, cn, NULL, vold, wold, u);
}

void ymom(double dt, double g, double r, double vb, Grid *grid, Visc *mu_old, Visc *mu_new,
          double ***cn, double ***uold, double ***wold, Velo *v)
{
    momentum(2, dt, g, r, vb, grid, mu_old, mu_new, cn, uold, NULL, wold, v);
}

void zmom(double dt, double g, double r, double vb, Grid *grid, Visc *mu_old, Visc *mu_new,
          double ***uold, double ***vold, Velo *w)
{
    momentum(3, dt, g, r, vb, grid, mu_old, mu_new, NULL, uold, vold, NULL, w);
}

/* update_velo_boundary L2701-2755 / update_veloghost_points L2810-2885 */
static void velo_ghosts(Grid *grid, Velo *u, Velo *v, Velo *w)
{
    if (!ctx_for(grid)) return;
    if (up(grid, PLLGPU_U_NEW, u->next) || up(grid, PLLGPU_V_NEW, v->next) || up(grid, PLLGPU_W_NEW, w->next))
        return;
    if (run(PLLGPU_R_VELO_GHOSTS, 0, 0, 0, 0, NULL)) return;
    down(grid, PLLGPU_U_NEW, u->next);
    down(grid, PLLGPU_V_NEW, v->next);
    down(grid, PLLGPU_W_NEW, w->next);
}

void update_velo_boundary(Grid *grid, Velo *u, Velo *v, Velo *w) { velo_ghosts(grid, u, v, w); }
void update_veloghost_points(Grid *grid, Velo *u, Velo *v, Velo *w) { velo_ghosts(grid, u, v, w); }

/* divergence, pllcart3d.c:1983-1999 */
void divergence(Grid *grid, double ***un, double ***vn, double ***wn, double ***div)
{
    if (!ctx_for(grid)) return;
    if (up(grid, PLLGPU_U_NEW, un) || up(grid, PLLGPU_V_NEW, vn) || up(grid, PLLGPU_W_NEW, wn) ||
        up(grid, PLLGPU_DIV, div))
        return;
    if (run(PLLGPU_R_DIVERGENCE, 0, 0, 0, 0, NULL)) return;
    down(grid, PLLGPU_DIV, div);
}

/* phisolver_dct, pllcart3d.c:2002-2130 */
void phisolver_dct(double dt, double g, double r, Grid *grid, double ***div, double ***phi)
{
    if (!ctx_for(grid)) return;
    if (up(grid, PLLGPU_DIV, div) || up(grid, PLLGPU_PHI, phi)) return;
    if (run(PLLGPU_R_PHISOLVER, dt, g, r, 0, NULL)) return;
    down(grid, PLLGPU_PHI, phi);
}

/* update_phi_ghosts, pllcart3d.c:2758-2807 */
void update_phi_ghosts(Grid *grid, double ***phi)
{
    if (!ctx_for(grid)) return;
    if (up(grid, PLLGPU_PHI, phi)) return;
    if (run(PLLGPU_R_PHI_GHOSTS, 0, 0, 0, 0, NULL)) return;
    down(grid, PLLGPU_PHI, phi);
}

/* velo_correction, pllcart3d.c:2133-2227 */
void velo_correction(double dt, double g, double r, Grid *grid, double ***phi, Velo *u, Velo *v, Velo *w)
{
    if (!ctx_for(grid)) return;
    if (up(grid, PLLGPU_PHI, phi) || up(grid, PLLGPU_U_NEW, u->next) || up(grid, PLLGPU_V_NEW, v->next) ||
        up(grid, PLLGPU_W_NEW, w->next))
        return;
    if (run(PLLGPU_R_VELO_CORRECTION, dt, g, r, 0, NULL)) return;
    down(grid, PLLGPU_U_NEW, u->next);
    down(grid, PLLGPU_V_NEW, v->next);
    down(grid, PLLGPU_W_NEW, w->next);
}

/* pressure_gradient, pllcart3d.c:2964-3044: A comes from the viscosity the
 * Tri_abc arrays were last built from (mu_new of the momentum routines) */
void pressure_gradient(double dt, double g, double r, Grid *grid, double ***phi, Velo *u, Velo *v, Velo *w)
{
    if (!ctx_for(grid)) return;
    if (!g_asrc[1] || g_asrc[1] != g_asrc[2] || g_asrc[1] != g_asrc[3]) {
        record(PLLGPU_EINVAL);
        return;
    }
    if (up(grid, PLLGPU_PHI, phi) || up(grid, PLLGPU_U_PG, u->pg) || up(grid, PLLGPU_V_PG, v->pg) ||
        up(grid, PLLGPU_W_PG, w->pg) || up_visc(grid, PLLGPU_MU_NEW_CELL, g_asrc[1]))
        return;
    if (run(PLLGPU_R_PRESSURE_GRADIENT, dt, g, r, 0, NULL)) return;
    down(grid, PLLGPU_U_PG, u->pg);
    down(grid, PLLGPU_V_PG, v->pg);
    down(grid, PLLGPU_W_PG, w->pg);
}

/* find_cfl, pllcart3d.c:3095-3118 (returns CFLmax / max) */
double find_cfl(Grid *grid, double ***un, double ***vn, double ***wn)
{
    double v = 0.0;
    if (!ctx_for(grid)) return v;
    if (up(grid, PLLGPU_U_OLD, un) || up(grid, PLLGPU_V_OLD, vn) || up(grid, PLLGPU_W_OLD, wn)) return v;
    run(PLLGPU_R_FIND_CFL, 0, 0, 0, 0, &v);
    return v;
}

/* bulk_velo, pllcart3d.c:3381-3398 */
double bulk_velo(Grid *grid, double ***un)
{
    double v = 0.0;
    if (!ctx_for(grid)) return v;
    if (up(grid, PLLGPU_U_OLD, un)) return v;
    run(PLLGPU_R_BULK_VELO, 0, 0, 0, 0, &v);
    return v;
}

/* update_old_conc / update_old_velo / update_old_visc (L3402-3452): the
 * copies go through the device buffers of the context */
static void copy_via_device(const Grid *g, int field, double ***src, double ***dst)
{
    if (up(g, field, src)) return;
    down(g, field, dst);
}

static Grid g_any; /* dimensions only, for the copies */

static Grid *grid_of(int nx_max, int ny_max, int nz_max)
{
    if (!g_ctx) return NULL;
    g_any.nx_max = nx_max;
    g_any.ny_max = ny_max;
    g_any.nz_max = nz_max;
    return &g_any;
}

void update_old_conc(Conc *c)
{
    Grid *g = grid_of(c->nx_max, c->ny_max, c->nz_max);
    if (!g) { record(PLLGPU_EINVAL); return; }
    copy_via_device(g, PLLGPU_C_NEW, c->next, c->old);
    copy_via_device(g, PLLGPU_C_HN, c->explicit_n, c->explicit_nm1);
}

void update_old_velo(Velo *u, Velo *v, Velo *w)
{
    Grid *g = grid_of(u->nx_max, u->ny_max, u->nz_max);
    Velo *q[3];
    int t;
    if (!g) { record(PLLGPU_EINVAL); return; }
    q[0] = u; q[1] = v; q[2] = w;
    for (t = 0; t < 3; t++) {
        copy_via_device(g, PLLGPU_U_NEW, q[t]->next, q[t]->old);
        copy_via_device(g, PLLGPU_U_HN, q[t]->explicit_n, q[t]->explicit_nm1);
    }
}

void update_old_visc(Visc *mu_old, Visc *mu_new)
{
    Grid *g = grid_of(mu_new->nx_max, mu_new->ny_max, mu_new->nz_max);
    if (!g) { record(PLLGPU_EINVAL); return; }
    copy_via_device(g, PLLGPU_MU_NEW_CELL, mu_new->cell, mu_old->cell);
    copy_via_device(g, PLLGPU_MU_NEW_XY, mu_new->xy, mu_old->xy);
    copy_via_device(g, PLLGPU_MU_NEW_XZ, mu_new->xz, mu_old->xz);
    copy_via_device(g, PLLGPU_MU_NEW_YZ, mu_new->yz, mu_old->yz);
}

/* calculate_weno, pllcart3d.c:3455-3507 */
double calculate_weno(double *d1, int kk, int sign)
{
    double v5[5], out = 0.0;
    int m;
    for (m = 0; m < 5; m++) v5[m] = d1[kk + sign * m];
    record(pllgpu_weno_batch(1, v5, &out));
    return out;
}

/* tridiag_1rhs, pllcart3d.c:3511-3536 */
int tridiag_1rhs(int Nmax, double *a, double *b, double *c, double *rhs)
{
    record(pllgpu_tridiag_1rhs_batch(1, Nmax, a, b, c, rhs));
    return 0;
}

/* pll_tridiag, pll_tridiag.c:152-158 (one rank): N systems of length n */
void pll_tridiag(Tds *arr, int N, int n)
{
    double *a, *b, *c, *r;
    int s;
    if (N <= 0 || n <= 0) return;
    a = (double *)malloc(sizeof(double) * (size_t)N * n * 4);
    if (!a) { record(PLLGPU_EINVAL); return; }
    b = a + (long)N * n;
    c = b + (long)N * n;
    r = c + (long)N * n;
    for (s = 0; s < N; s++) {
        memcpy(a + (long)s * n, arr[s].acof, sizeof(double) * n);
        memcpy(b + (long)s * n, arr[s].bcof, sizeof(double) * n);
        memcpy(c + (long)s * n, arr[s].ccof, sizeof(double) * n);
        memcpy(r + (long)s * n, arr[s].rhs, sizeof(double) * n);
    }
    if (!record(pllgpu_tridiag_batch(N, n, a, b, c, r))) {
        for (s = 0; s < N; s++) {
            memcpy(arr[s].bcof, b + (long)s * n, sizeof(double) * n);
            memcpy(arr[s].ccof, c + (long)s * n, sizeof(double) * n);
            memcpy(arr[s].rhs, r + (long)s * n, sizeof(double) * n);
        }
    }
    free(a);
}

/* plan_dct_3d / fdct_3d / idct_3d, fftw_3d.h:12-106: datain[i][j][k] with
 * i < ndim1, j < ndim2, k < num_transforms; transform k is the ndim2 x ndim1
 * array DCT_in[k*N + j*N1 + i] */
void plan_dct_3d(int ndim1, int ndim2, int num_transforms)
{
    g_dct_n1 = ndim1;
    g_dct_n2 = ndim2;
    g_dct_nt = num_transforms;
}

static void dct_3d(int inverse, int ndim1, int ndim2, int nt, double ***datain, double ***dataout)
{
    long N = (long)ndim1 * ndim2;
    double *x = (double *)malloc(sizeof(double) * (size_t)N * nt * 2), *y;
    int i, j, k, e;
    if (!x) { record(PLLGPU_EINVAL); return; }
    y = x + N * nt;
    for (k = 0; k < nt; k++)
        for (j = 0; j < ndim2; j++)
            for (i = 0; i < ndim1; i++) x[k * N + (long)j * ndim1 + i] = datain[i][j][k];
    e = inverse ? pllgpu_idct2d_batch(ndim2, ndim1, nt, x, y) : pllgpu_dct2d_batch(0, ndim2, ndim1, nt, x, y);
    if (!record(e))
        for (k = 0; k < nt; k++)
            for (j = 0; j < ndim2; j++)
                for (i = 0; i < ndim1; i++) dataout[i][j][k] = y[k * N + (long)j * ndim1 + i];
    free(x);
}

void fdct_3d(int ndim1, int ndim2, int nt, double ***datain, double ***dataout)
{
    dct_3d(0, ndim1, ndim2, nt, datain, dataout);
}

void idct_3d(int ndim1, int ndim2, int nt, double ***datain, double ***dataout)
{
    dct_3d(1, ndim1, ndim2, nt, datain, dataout);
}

/* ---- resident fast path ---------------------------------------------- */

/* upload the whole state after the host's own start-up
 * (pllcart3d.c:57-154) */
int pllgpu_attach(Grid *grid, Velo *u, Velo *v, Velo *w, Conc *c, Visc *mu_old, Visc *mu_new, double ***phi)
{
    int e = 0, t;
    Velo *q[3];
    static const int base[3] = {PLLGPU_U_OLD, PLLGPU_V_OLD, PLLGPU_W_OLD};
    if (!ctx_for(grid)) return g_status;
    a_grid = grid; a_u = u; a_v = v; a_w = w; a_c = c; a_mu_old = mu_old; a_mu_new = mu_new; a_phi = phi;
    q[0] = u; q[1] = v; q[2] = w;
    e = e || up(grid, PLLGPU_C_OLD, c->old) || up(grid, PLLGPU_C_NEW, c->next) ||
        up(grid, PLLGPU_C_HN, c->explicit_n) || up(grid, PLLGPU_C_HNM1, c->explicit_nm1);
    for (t = 0; t < 3 && !e; t++)
        e = up(grid, base[t] + 0, q[t]->old) || up(grid, base[t] + 1, q[t]->next) ||
            up(grid, base[t] + 2, q[t]->explicit_n) || up(grid, base[t] + 3, q[t]->explicit_nm1) ||
            up(grid, base[t] + 4, q[t]->pg);
    e = e || up_visc(grid, PLLGPU_MU_OLD_CELL, mu_old) || up_visc(grid, PLLGPU_MU_NEW_CELL, mu_new) ||
        up(grid, PLLGPU_PHI, phi);
    if (!e) e = record(pllgpu_set_timestep(g_ctx, Timestep));
    return e ? g_status : PLLGPU_OK;
}

/* nsteps time steps of pllcart3d.c:158-195 on the device; *tval advanced */
int pllgpu_advance(int nsteps, double *tval)
{
    int e;
    if (!g_ctx || !a_grid) return record(PLLGPU_EINVAL);
    if (tval && (e = record(pllgpu_set_tval(g_ctx, *tval)))) return e;
    if ((e = record(pllgpu_steps(g_ctx, nsteps)))) return e;
    if (tval) *tval = pllgpu_tval(g_ctx);
    return PLLGPU_OK;
}

/* the device context behind pllgpu_attach, for the resident output calls
 * (pllgpu_write_snapshot, pllgpu_write_restart, pllgpu_conc_average,
 * pllgpu_find_max, pllgpu_find_wmax, pllgpu_shift_conc) that replace the
 * reference's file output without a copy of the state to the host */
pllgpu_ctx *pllgpu_dropin_context(void) { return g_ctx; }

/* state back into the attached host arrays (before any of the reference's
 * file output or diagnostics, pllcart3d.c:198-256) */
int pllgpu_sync_to_host(void)
{
    int e = 0, t;
    Velo *q[3];
    static const int base[3] = {PLLGPU_U_OLD, PLLGPU_V_OLD, PLLGPU_W_OLD};
    Grid *g = a_grid;
    if (!g_ctx || !g) return record(PLLGPU_EINVAL);
    q[0] = a_u; q[1] = a_v; q[2] = a_w;
    e = e || down(g, PLLGPU_C_OLD, a_c->old) || down(g, PLLGPU_C_NEW, a_c->next) ||
        down(g, PLLGPU_C_HN, a_c->explicit_n) || down(g, PLLGPU_C_HNM1, a_c->explicit_nm1);
    for (t = 0; t < 3 && !e; t++) {
        e = down(g, base[t] + 0, q[t]->old) || down(g, base[t] + 1, q[t]->next) ||
            down(g, base[t] + 2, q[t]->explicit_n) || down(g, base[t] + 3, q[t]->explicit_nm1) ||
            down(g, base[t] + 4, q[t]->pg);
    }
    e = e || down_visc(g, PLLGPU_MU_OLD_CELL, a_mu_old) || down_visc(g, PLLGPU_MU_NEW_CELL, a_mu_new) ||
        down(g, PLLGPU_PHI, a_phi);
    if (!e) {
        /* Tri_abc arrays as the last substep left them: A(mu_new) */
        for (t = 0; t < 3; t++)
            fill_abc(g, t + 1, q[t]->istart, q[t]->iend, q[t]->jstart, q[t]->jend, q[t]->kstart, q[t]->kend,
                     q[t]->Ax, q[t]->Ay, q[t]->Az);
        g_asrc[1] = g_asrc[2] = g_asrc[3] = a_mu_new;
    }
    return e ? g_status : PLLGPU_OK;
}

void pllgpu_finalize(void)
{
    if (g_ctx) pllgpu_destroy(g_ctx);
    g_ctx = NULL;
    free(g_stage);
    free(g_abc);
    g_stage = NULL;
    g_abc = NULL;
}
