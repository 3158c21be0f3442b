/*
 * Driver around the reference's own step routines (compiled from
 * pllcart3d.c / pll_tridiag.c into oracle/_ref/ by oracle/Makefile).
 * Test infrastructure only: it exists so that the CPU restatement in
 * oracle/pllcart3d_oracle.c can be pinned against the reference itself and so
 * that the reference CPU path can be timed.  It is never part of the GPU
 * library.
 *
 * pllref_init mirrors main() start-up (pllcart3d.c:57-73); pllref_load_ic
 * replaces initial_condition (pllcart3d.c:80) by caller-supplied arrays and
 * then runs pllcart3d.c:81-83 and 126-154; pllref_steps runs the time-step
 * body pllcart3d.c:158-195 a fixed number of times (diagnostics and file
 * output of pllcart3d.c:198-256 are left out).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "structures_3d.h"

/* reference globals (global_variables.h, pllcart3d.c:36) */
extern int Nx_cell_global, Ny_cell_global, Nz_cell_global;
extern int Nx_ghost, Ny_ghost, Nz_ghost;
extern int Initial, Ugrid, Niter_print, Wavpert, Subharm, Nmvp;
extern double X1, X2, Y1, Y2, Z1, Z2;
extern double Re, Pe, Vratio, Fx, Fy, Inf_pos, Inf_thick;
extern double CFLmax, Timemax, Timestep, Out_inter, Out_mid;
extern double PI, M, Vnorm, Ampli, Lamb, Mum, Lambda;
extern double RK1[3], RK2[3];
extern int Rank, Size;

/* reference routines (global_function_decl.h, allocate_3d_calloc.h) */
void input();
void grid_setup(Grid *);
void simulation_setup(Grid *, Velo *, Velo *, Velo *, Conc *);
void mesh_generation(Grid *);
void plan_dct_3d(int, int, int);
void fdct_3d(int, int, int, double ***, double ***);
void idct_3d(int, int, int, double ***, double ***);
Velo *alloc_velo(int, int, int);
Conc *alloc_conc(int, int, int);
Visc *alloc_visc(int, int, int);
double ***alloc3d_dble(int, int, int);
Tds *alloc_tds(int, int);
void free_tds(Tds *, int, int);
void pll_tridiag(Tds *, int, int);
int tridiag_1rhs(int, double *, double *, double *, double *);
double calculate_weno(double *, int, int);
void concentration(double, double, double, double, Grid *, double ***,
                   double ***, double ***, Conc *);
double slope_parameter(Grid *, double ***);
void calculate_viscosity(Grid *, double ***, Visc *);
void calculate_viscosity_nmvp(Grid *, double ***, Visc *, double);
void xmom(double, double, double, double, Grid *, Visc *, Visc *, double ***,
          double ***, double ***, Velo *);
void ymom(double, double, double, double, Grid *, Visc *, Visc *, double ***,
          double ***, double ***, Velo *);
void zmom(double, double, double, double, Grid *, Visc *, Visc *, double ***,
          double ***, Velo *);
void A_conc(Grid *, Conc *);
void A_umom(Grid *, Visc *, Velo *);
void A_vmom(Grid *, Visc *, Velo *);
void A_wmom(Grid *, Visc *, Velo *);
void divergence(Grid *, double ***, double ***, double ***, double ***);
void phisolver_dct(double, double, double, Grid *, double ***, double ***);
void velo_correction(double, double, double, Grid *, double ***, Velo *,
                     Velo *, Velo *);
void update_veloghost_points(Grid *, Velo *, Velo *, Velo *);
void update_ghost_points(Grid *, double ***, Velo *, Velo *, Velo *);
void update_velo_boundary(Grid *, Velo *, Velo *, Velo *);
void update_phi_ghosts(Grid *, double ***);
void pressure_gradient(double, double, double, Grid *, double ***, Velo *,
                       Velo *, Velo *);
double find_cfl(Grid *, double ***, double ***, double ***);
double bulk_velo(Grid *, double ***);
void update_old_conc(Conc *);
void update_old_velo(Velo *, Velo *, Velo *);
void update_old_visc(Visc *, Visc *);
void pll_shim_fftw_set_fast(int);
void write_to_file(int, Grid *, double ***, double ***, double ***, double ***);
void midfield(int, int, double, double, double, double, Grid *, Conc *, Velo *, Velo *, Velo *);
void intermediate(int *, int *, double *, double *, Grid *, Conc *, Velo *, Velo *, Velo *);
void conc_average(Grid *, double ***, double);
void find_wmax(double, Grid *, Velo *);
void find_max(Grid *, Velo *, Velo *, Velo *, Conc *);
void shift_conc(Grid *, Conc *);

static Grid *g_grid;
static Velo *g_u, *g_v, *g_w;
static Conc *g_c;
static Visc *g_mu_old, *g_mu_new;
static double ***g_phi, ***g_div;
static double g_tval, g_dt, g_cm;
static char g_rundir[4096]; /* where the reference's side files go */

/* set-up of rank `rank` of `size` (pllcart3d.c:57-80 up to the initial
 * condition); pllref_init is the single-rank case */
int pllref_init_ranked(const char *rundir, int rank, int size)
{
    char here[4096];
    if (!getcwd(here, sizeof(here))) return -1;
    if (chdir(rundir) != 0) return -1;
    strncpy(g_rundir, rundir, sizeof(g_rundir) - 1);
    Rank = rank;
    Size = size;
    input();
    g_grid = (Grid *)malloc(sizeof(Grid));
    grid_setup(g_grid);
    g_u = alloc_velo(g_grid->nx_max, g_grid->ny_max, g_grid->nz_max);
    g_v = alloc_velo(g_grid->nx_max, g_grid->ny_max, g_grid->nz_max);
    g_w = alloc_velo(g_grid->nx_max, g_grid->ny_max, g_grid->nz_max);
    g_c = alloc_conc(g_grid->nx_max, g_grid->ny_max, g_grid->nz_max);
    g_mu_old = alloc_visc(g_grid->nx_max, g_grid->ny_max, g_grid->nz_max);
    g_mu_new = alloc_visc(g_grid->nx_max, g_grid->ny_max, g_grid->nz_max);
    g_phi = alloc3d_dble(g_grid->nx_max, g_grid->ny_max, g_grid->nz_max);
    g_div = alloc3d_dble(g_grid->nx_max, g_grid->ny_max, g_grid->nz_max);
    simulation_setup(g_grid, g_u, g_v, g_w, g_c);
    mesh_generation(g_grid);
    plan_dct_3d(g_grid->ny_cell, g_grid->nz_cell, g_grid->nx_cell);
    g_tval = 0.0;
    if (chdir(here) != 0) return -1;
    return 0;
}

int pllref_init(const char *rundir) { return pllref_init_ranked(rundir, 0, 1); }

/* first global x cell of this rank's slab (grid_setup, pllcart3d.c:376-379) */
int pllref_x_offset(void) { return g_grid->nx_global_offset; }

/* input() (pllcart3d.c:271-350) on <dir>/param.input; its 34 values in
 * file order, as doubles, into out[34] */
int pllref_read_input(const char *dir, double *out)
{
    char here[4096];
    int n = 0;
    if (!getcwd(here, sizeof(here)) || chdir(dir) != 0) return -1;
    input();
    if (chdir(here) != 0) return -1;
    out[n++] = Nx_cell_global; out[n++] = Ny_cell_global; out[n++] = Nz_cell_global;
    out[n++] = Nx_ghost; out[n++] = Ny_ghost; out[n++] = Nz_ghost;
    out[n++] = Initial; out[n++] = Ugrid; out[n++] = Niter_print; out[n++] = Out_mid;
    out[n++] = X1; out[n++] = X2; out[n++] = Y1; out[n++] = Y2; out[n++] = Z1; out[n++] = Z2;
    out[n++] = Timemax; out[n++] = Timestep; out[n++] = Re; out[n++] = Pe; out[n++] = Vratio;
    out[n++] = Fx; out[n++] = Fy; out[n++] = Inf_pos; out[n++] = Inf_thick; out[n++] = CFLmax;
    out[n++] = Out_inter; out[n++] = Wavpert; out[n++] = Ampli; out[n++] = Lamb; out[n++] = Subharm;
    out[n++] = Nmvp; out[n++] = Mum; out[n++] = Lambda;
    return n;
}

void pllref_set_fast_dct(int fast) { pll_shim_fftw_set_fast(fast); }

void pllref_dims(int *d)
{
    d[0] = g_grid->nx_max;
    d[1] = g_grid->ny_max;
    d[2] = g_grid->nz_max;
    d[3] = g_grid->nx_cell;
    d[4] = g_grid->ny_cell;
    d[5] = g_grid->nz_cell;
}

static double ***field(const char *name)
{
    if (!strcmp(name, "c_old")) return g_c->old;
    if (!strcmp(name, "c_new")) return g_c->new;
    if (!strcmp(name, "c_hn")) return g_c->explicit_n;
    if (!strcmp(name, "c_hnm1")) return g_c->explicit_nm1;
#define VEL(P, V)                                                   \
    if (!strcmp(name, P "_old")) return V->old;                     \
    if (!strcmp(name, P "_new")) return V->new;                     \
    if (!strcmp(name, P "_hn")) return V->explicit_n;               \
    if (!strcmp(name, P "_hnm1")) return V->explicit_nm1;           \
    if (!strcmp(name, P "_pg")) return V->pg;
    VEL("u", g_u)
    VEL("v", g_v)
    VEL("w", g_w)
#undef VEL
#define MU(P, V)                                                    \
    if (!strcmp(name, P "_cell")) return V->cell;                   \
    if (!strcmp(name, P "_xy")) return V->xy;                       \
    if (!strcmp(name, P "_xz")) return V->xz;                       \
    if (!strcmp(name, P "_yz")) return V->yz;
    MU("mu_old", g_mu_old)
    MU("mu_new", g_mu_new)
#undef MU
    if (!strcmp(name, "phi")) return g_phi;
    if (!strcmp(name, "div")) return g_div;
    return NULL;
}

static Tri_abc ***abc_field(const char *name)
{
    if (!strcmp(name, "c_Ax")) return g_c->Ax;
    if (!strcmp(name, "c_Ay")) return g_c->Ay;
    if (!strcmp(name, "c_Az")) return g_c->Az;
    if (!strcmp(name, "u_Ax")) return g_u->Ax;
    if (!strcmp(name, "u_Ay")) return g_u->Ay;
    if (!strcmp(name, "u_Az")) return g_u->Az;
    if (!strcmp(name, "v_Ax")) return g_v->Ax;
    if (!strcmp(name, "v_Ay")) return g_v->Ay;
    if (!strcmp(name, "v_Az")) return g_v->Az;
    if (!strcmp(name, "w_Ax")) return g_w->Ax;
    if (!strcmp(name, "w_Ay")) return g_w->Ay;
    if (!strcmp(name, "w_Az")) return g_w->Az;
    return NULL;
}

int pllref_get(const char *name, double *out)
{
    int i, j, NY = g_grid->ny_max, NZ = g_grid->nz_max;
    double ***f = field(name);
    if (!f) return -1;
    for (i = 0; i < g_grid->nx_max; i++)
        for (j = 0; j < NY; j++)
            memcpy(out + ((long)i * NY + j) * NZ, f[i][j], sizeof(double) * NZ);
    return 0;
}

int pllref_set(const char *name, const double *in)
{
    int i, j, NY = g_grid->ny_max, NZ = g_grid->nz_max;
    double ***f = field(name);
    if (!f) return -1;
    for (i = 0; i < g_grid->nx_max; i++)
        for (j = 0; j < NY; j++)
            memcpy(f[i][j], in + ((long)i * NY + j) * NZ, sizeof(double) * NZ);
    return 0;
}

/* coefficient triples on the variable's own interior range only (the rest of
 * a Tri_abc row is uninitialised malloc memory, allocate_3d_calloc.h:97) */
int pllref_get_abc(const char *name, int is, int ie, int js, int je, int ks,
                   int ke, double *a, double *b, double *c)
{
    int i, j, k, NY = g_grid->ny_max, NZ = g_grid->nz_max;
    Tri_abc ***f = abc_field(name);
    if (!f) return -1;
    for (i = is; i <= ie; i++)
        for (j = js; j <= je; j++)
            for (k = ks; k <= ke; k++) {
                long id = ((long)i * NY + j) * NZ + k;
                a[id] = f[i][j][k].a;
                b[id] = f[i][j][k].b;
                c[id] = f[i][j][k].c;
            }
    return 0;
}

/* A_conc / A_umom / A_vmom / A_wmom (pllcart3d.c:1411-1536) on the
 * reference's own structures, from the old (mu_which 0) or new (1)
 * viscosity, each taken from f[0..3] when given (the drop-in layer's) or
 * the reference's own.  Before the call the interior of every Tri_abc is
 * filled with NaN, so a coefficient the called routine does not write shows. */
typedef void (*ac_fn)(Grid *, Conc *);
typedef void (*am_fn)(Grid *, Visc *, Velo *);

static void nan_abc(Tri_abc ***f, int is, int ie, int js, int je, int ks, int ke)
{
    int i, j, k;
    for (i = is; i <= ie; i++)
        for (j = js; j <= je; j++)
            for (k = ks; k <= ke; k++) f[i][j][k].a = f[i][j][k].b = f[i][j][k].c = NAN;
}

int pllref_acoef_with(void **f, int mu_which)
{
    Visc *mu = mu_which ? g_mu_new : g_mu_old;
    ac_fn fc = (f && f[0]) ? (ac_fn)f[0] : A_conc;
    am_fn fu = (f && f[1]) ? (am_fn)f[1] : A_umom;
    am_fn fv = (f && f[2]) ? (am_fn)f[2] : A_vmom;
    am_fn fw = (f && f[3]) ? (am_fn)f[3] : A_wmom;
    nan_abc(g_c->Ax, g_c->istart, g_c->iend, g_c->jstart, g_c->jend, g_c->kstart, g_c->kend);
    nan_abc(g_c->Ay, g_c->istart, g_c->iend, g_c->jstart, g_c->jend, g_c->kstart, g_c->kend);
    nan_abc(g_c->Az, g_c->istart, g_c->iend, g_c->jstart, g_c->jend, g_c->kstart, g_c->kend);
#define NAN3(q) \
    nan_abc(q->Ax, q->istart, q->iend, q->jstart, q->jend, q->kstart, q->kend); \
    nan_abc(q->Ay, q->istart, q->iend, q->jstart, q->jend, q->kstart, q->kend); \
    nan_abc(q->Az, q->istart, q->iend, q->jstart, q->jend, q->kstart, q->kend)
    NAN3(g_u);
    NAN3(g_v);
    NAN3(g_w);
#undef NAN3
    fc(g_grid, g_c);
    fu(g_grid, mu, g_u);
    fv(g_grid, mu, g_v);
    fw(g_grid, mu, g_w);
    return 0;
}

/* the unknown range of a variable (0 c, 1 u, 2 v, 3 w): is, ie, js, je, ks, ke */
int pllref_range(int var, int *r)
{
    Conc *c = g_c;
    Velo *q = var == 1 ? g_u : var == 2 ? g_v : g_w;
    if (var == 0) {
        r[0] = c->istart; r[1] = c->iend; r[2] = c->jstart; r[3] = c->jend; r[4] = c->kstart; r[5] = c->kend;
    } else {
        r[0] = q->istart; r[1] = q->iend; r[2] = q->jstart; r[3] = q->jend; r[4] = q->kstart; r[5] = q->kend;
    }
    return 0;
}

/* pllcart3d.c:81-83 and 126-154 after caller-supplied initial fields */
int pllref_load_ic(const double *c, const double *u, const double *v,
                   const double *w)
{
    double del_min, diff_dt;
    char here[4096];
    /* slope_parameter appends to Outscreen in the working directory */
    if (!getcwd(here, sizeof(here)) || chdir(g_rundir) != 0) return -1;
    pllref_set("c_new", c);
    pllref_set("u_new", u);
    pllref_set("v_new", v);
    pllref_set("w_new", w);
    update_ghost_points(g_grid, g_phi, g_u, g_v, g_w);
    update_old_conc(g_c);
    update_old_velo(g_u, g_v, g_w);
    if (Nmvp == 1) {
        g_cm = slope_parameter(g_grid, g_c->new);
        calculate_viscosity_nmvp(g_grid, g_c->old, g_mu_old, g_cm);
    } else {
        calculate_viscosity(g_grid, g_c->old, g_mu_old);
    }
    A_conc(g_grid, g_c);
    A_umom(g_grid, g_mu_old, g_u);
    A_vmom(g_grid, g_mu_old, g_v);
    A_wmom(g_grid, g_mu_old, g_w);
    del_min = (g_grid->dx < g_grid->dy) ? g_grid->dx : g_grid->dy;
    del_min = (del_min < g_grid->dz) ? del_min : g_grid->dz;
    diff_dt = 0.1 * Pe * del_min * del_min;
    Timestep = (diff_dt < Timestep) ? diff_dt : Timestep;
    g_tval = 0.0;
    if (chdir(here) != 0) return -1;
    return 0;
}

/* pllcart3d.c:126-154 after intermediate() (L111) restored the state */
int pllref_restart_startup(double tval)
{
    double del_min, diff_dt;
    char here[4096];
    if (!getcwd(here, sizeof(here)) || chdir(g_rundir) != 0) return -1;
    if (Nmvp == 1) {
        g_cm = slope_parameter(g_grid, g_c->new);
        calculate_viscosity_nmvp(g_grid, g_c->old, g_mu_old, g_cm);
    } else {
        calculate_viscosity(g_grid, g_c->old, g_mu_old);
    }
    A_conc(g_grid, g_c);
    A_umom(g_grid, g_mu_old, g_u);
    A_vmom(g_grid, g_mu_old, g_v);
    A_wmom(g_grid, g_mu_old, g_w);
    del_min = (g_grid->dx < g_grid->dy) ? g_grid->dx : g_grid->dy;
    del_min = (del_min < g_grid->dz) ? del_min : g_grid->dz;
    diff_dt = 0.1 * Pe * del_min * del_min;
    Timestep = (diff_dt < Timestep) ? diff_dt : Timestep;
    g_tval = tval;
    if (chdir(here) != 0) return -1;
    return 0;
}

/* one RK3-CN substep, pllcart3d.c:164-194 */
void pllref_substep(double dt, int rkstep)
{
    double g = RK1[rkstep], r = RK2[rkstep], vbulk = 0.0;
    g_tval = g_tval + (g + r) * dt;
    vbulk = bulk_velo(g_grid, g_u->old);
    concentration(dt, g, r, vbulk, g_grid, g_u->new, g_v->new, g_w->new, g_c);
    if (Nmvp == 1)
        calculate_viscosity_nmvp(g_grid, g_c->new, g_mu_new, g_cm);
    else
        calculate_viscosity(g_grid, g_c->new, g_mu_new);
    xmom(dt, g, r, vbulk, g_grid, g_mu_old, g_mu_new, g_c->new, g_v->old,
         g_w->old, g_u);
    ymom(dt, g, r, vbulk, g_grid, g_mu_old, g_mu_new, g_c->new, g_u->old,
         g_w->old, g_v);
    zmom(dt, g, r, vbulk, g_grid, g_mu_old, g_mu_new, g_u->old, g_v->old, g_w);
    update_velo_boundary(g_grid, g_u, g_v, g_w);
    divergence(g_grid, g_u->new, g_v->new, g_w->new, g_div);
    phisolver_dct(dt, g, r, g_grid, g_div, g_phi);
    update_phi_ghosts(g_grid, g_phi);
    velo_correction(dt, g, r, g_grid, g_phi, g_u, g_v, g_w);
    update_veloghost_points(g_grid, g_u, g_v, g_w);
    pressure_gradient(dt, g, r, g_grid, g_phi, g_u, g_v, g_w);
    update_old_conc(g_c);
    update_old_velo(g_u, g_v, g_w);
    update_old_visc(g_mu_old, g_mu_new);
}

double pllref_step_dt(void)
{
    double cfl_dt = find_cfl(g_grid, g_u->old, g_v->old, g_w->old);
    return (cfl_dt < Timestep) ? cfl_dt : Timestep;
}

/* pllcart3d.c:158-195, n times */
int pllref_steps(int n)
{
    int s, rk;
    for (s = 0; s < n; s++) {
        g_dt = pllref_step_dt();
        for (rk = 0; rk < 3; rk++) pllref_substep(g_dt, rk);
    }
    return 0;
}

double pllref_last_dt(void) { return g_dt; }
double pllref_tval(void) { return g_tval; }
double pllref_timestep(void) { return Timestep; }

/* single routines, for per-routine parity */
void pllref_concentration(double dt, double g, double r, double vb)
{
    concentration(dt, g, r, vb, g_grid, g_u->new, g_v->new, g_w->new, g_c);
}
void pllref_viscosity_new(void) { calculate_viscosity(g_grid, g_c->new, g_mu_new); }
void pllref_xmom(double dt, double g, double r, double vb)
{
    xmom(dt, g, r, vb, g_grid, g_mu_old, g_mu_new, g_c->new, g_v->old, g_w->old, g_u);
}
void pllref_ymom(double dt, double g, double r, double vb)
{
    ymom(dt, g, r, vb, g_grid, g_mu_old, g_mu_new, g_c->new, g_u->old, g_w->old, g_v);
}
void pllref_zmom(double dt, double g, double r, double vb)
{
    zmom(dt, g, r, vb, g_grid, g_mu_old, g_mu_new, g_u->old, g_v->old, g_w);
}
void pllref_update_velo_boundary(void) { update_velo_boundary(g_grid, g_u, g_v, g_w); }
void pllref_divergence(void) { divergence(g_grid, g_u->new, g_v->new, g_w->new, g_div); }
void pllref_phisolver(double dt, double g, double r) { phisolver_dct(dt, g, r, g_grid, g_div, g_phi); }
void pllref_update_phi_ghosts(void) { update_phi_ghosts(g_grid, g_phi); }
void pllref_velo_correction(double dt, double g, double r)
{
    velo_correction(dt, g, r, g_grid, g_phi, g_u, g_v, g_w);
}
void pllref_update_veloghost_points(void) { update_veloghost_points(g_grid, g_u, g_v, g_w); }
void pllref_pressure_gradient(double dt, double g, double r)
{
    pressure_gradient(dt, g, r, g_grid, g_phi, g_u, g_v, g_w);
}
void pllref_rotate(void)
{
    update_old_conc(g_c);
    update_old_velo(g_u, g_v, g_w);
    update_old_visc(g_mu_old, g_mu_new);
}
void pllref_rebuild_A_old(void)
{
    A_umom(g_grid, g_mu_old, g_u);
    A_vmom(g_grid, g_mu_old, g_v);
    A_wmom(g_grid, g_mu_old, g_w);
}
double pllref_find_cfl(void) { return find_cfl(g_grid, g_u->old, g_v->old, g_w->old); }
double pllref_bulk_velo(void) { return bulk_velo(g_grid, g_u->old); }

/* batched line solves through the reference's pll_tridiag / tridiag_1rhs */
void pllref_pll_tridiag(int N, int n, double *a, double *b, double *c, double *r)
{
    int s;
    Tds *t = alloc_tds(N, n);
    for (s = 0; s < N; s++) {
        memcpy(t[s].acof, a + (long)s * n, sizeof(double) * n);
        memcpy(t[s].bcof, b + (long)s * n, sizeof(double) * n);
        memcpy(t[s].ccof, c + (long)s * n, sizeof(double) * n);
        memcpy(t[s].rhs, r + (long)s * n, sizeof(double) * n);
    }
    pll_tridiag(t, N, n);
    for (s = 0; s < N; s++) {
        memcpy(b + (long)s * n, t[s].bcof, sizeof(double) * n);
        memcpy(c + (long)s * n, t[s].ccof, sizeof(double) * n);
        memcpy(r + (long)s * n, t[s].rhs, sizeof(double) * n);
    }
    free_tds(t, N, n);
}
int pllref_tridiag_1rhs(int n, double *a, double *b, double *c, double *r)
{
    return tridiag_1rhs(n, a, b, c, r);
}
double pllref_calculate_weno(double *d1, int kk, int sign)
{
    return calculate_weno(d1, kk, sign);
}

/* The time-step loop of pllcart3d.c:158-195 with any of its routines taken
 * from a table of replacements (NULL entries keep the reference's own):
 * 0 concentration 1 calculate_viscosity 2 xmom 3 ymom 4 zmom
 * 5 update_velo_boundary 6 divergence 7 phisolver_dct 8 update_phi_ghosts
 * 9 velo_correction 10 update_veloghost_points 11 pressure_gradient
 * 12 update_old_conc 13 update_old_velo 14 update_old_visc 15 find_cfl
 * 16 bulk_velo.  Used to run the drop-in layer inside the reference's own
 * loop, on the reference's own structures. */
typedef void (*conc_fn)(double, double, double, double, Grid *, double ***, double ***, double ***, Conc *);
typedef void (*visc_fn)(Grid *, double ***, Visc *);
typedef void (*mom_fn)(double, double, double, double, Grid *, Visc *, Visc *, double ***, double ***,
                       double ***, Velo *);
typedef void (*zmom_fn)(double, double, double, double, Grid *, Visc *, Visc *, double ***, double ***, Velo *);
typedef void (*vb_fn)(Grid *, Velo *, Velo *, Velo *);
typedef void (*div_fn)(Grid *, double ***, double ***, double ***, double ***);
typedef void (*phi_fn)(double, double, double, Grid *, double ***, double ***);
typedef void (*phig_fn)(Grid *, double ***);
typedef void (*corr_fn)(double, double, double, Grid *, double ***, Velo *, Velo *, Velo *);
typedef void (*oc_fn)(Conc *);
typedef void (*ov_fn)(Velo *, Velo *, Velo *);
typedef void (*om_fn)(Visc *, Visc *);
typedef double (*cfl_fn)(Grid *, double ***, double ***, double ***);
typedef double (*bulk_fn)(Grid *, double ***);

int pllref_steps_with(int n, void **f)
{
    int s, rk;
#define PICK(i, T, dflt) ((f && f[i]) ? (T)f[i] : (T)dflt)
    conc_fn f_conc = PICK(0, conc_fn, concentration);
    visc_fn f_visc = PICK(1, visc_fn, calculate_viscosity);
    mom_fn f_x = PICK(2, mom_fn, xmom), f_y = PICK(3, mom_fn, ymom);
    zmom_fn f_z = PICK(4, zmom_fn, zmom);
    vb_fn f_vb = PICK(5, vb_fn, update_velo_boundary);
    div_fn f_div = PICK(6, div_fn, divergence);
    phi_fn f_phi = PICK(7, phi_fn, phisolver_dct);
    phig_fn f_phig = PICK(8, phig_fn, update_phi_ghosts);
    corr_fn f_corr = PICK(9, corr_fn, velo_correction);
    vb_fn f_vg = PICK(10, vb_fn, update_veloghost_points);
    corr_fn f_pg = PICK(11, corr_fn, pressure_gradient);
    oc_fn f_oc = PICK(12, oc_fn, update_old_conc);
    ov_fn f_ov = PICK(13, ov_fn, update_old_velo);
    om_fn f_om = PICK(14, om_fn, update_old_visc);
    cfl_fn f_cfl = PICK(15, cfl_fn, find_cfl);
    bulk_fn f_bulk = PICK(16, bulk_fn, bulk_velo);
#undef PICK
    for (s = 0; s < n; s++) {
        double cfl_dt = f_cfl(g_grid, g_u->old, g_v->old, g_w->old);
        g_dt = (cfl_dt < Timestep) ? cfl_dt : Timestep;
        for (rk = 0; rk < 3; rk++) {
            double g = RK1[rk], r = RK2[rk], vbulk;
            g_tval = g_tval + (g + r) * g_dt;
            vbulk = f_bulk(g_grid, g_u->old);
            f_conc(g_dt, g, r, vbulk, g_grid, g_u->new, g_v->new, g_w->new, g_c);
            f_visc(g_grid, g_c->new, g_mu_new);
            f_x(g_dt, g, r, vbulk, g_grid, g_mu_old, g_mu_new, g_c->new, g_v->old, g_w->old, g_u);
            f_y(g_dt, g, r, vbulk, g_grid, g_mu_old, g_mu_new, g_c->new, g_u->old, g_w->old, g_v);
            f_z(g_dt, g, r, vbulk, g_grid, g_mu_old, g_mu_new, g_u->old, g_v->old, g_w);
            f_vb(g_grid, g_u, g_v, g_w);
            f_div(g_grid, g_u->new, g_v->new, g_w->new, g_div);
            f_phi(g_dt, g, r, g_grid, g_div, g_phi);
            f_phig(g_grid, g_phi);
            f_corr(g_dt, g, r, g_grid, g_phi, g_u, g_v, g_w);
            f_vg(g_grid, g_u, g_v, g_w);
            f_pg(g_dt, g, r, g_grid, g_phi, g_u, g_v, g_w);
            f_oc(g_c);
            f_ov(g_u, g_v, g_w);
            f_om(g_mu_old, g_mu_new);
        }
    }
    return 0;
}

/* the reference's own structures, for hosts that hand them to another
 * implementation (the resident GPU path) */
void pllref_structs(void **out)
{
    out[0] = g_grid; out[1] = g_u; out[2] = g_v; out[3] = g_w; out[4] = g_c;
    out[5] = g_mu_old; out[6] = g_mu_new; out[7] = g_phi;
}

void pllref_set_tval(double t) { g_tval = t; }

/* ---- the reference's own output routines, run in `dir` ------------------
 * write_to_file pllcart3d.c:3047, midfield L3121, intermediate L3181,
 * conc_average L3635, find_wmax L3606, find_max L3539 (whose NaN branch
 * calls exit(1); callers only use it on finite states). */
static int in_dir(const char *dir, char *here)
{
    if (!getcwd(here, 4096)) return -1;
    return chdir(dir);
}

int pllref_write_to_file(int fileno, const char *dir)
{
    char here[4096];
    if (in_dir(dir, here)) return -1;
    write_to_file(fileno, g_grid, g_u->new, g_v->new, g_w->new, g_c->new);
    return chdir(here);
}

int pllref_midfield(int tstep, int fileno, double tval, double outtime, double outmid, double cavgtime,
                    const char *dir)
{
    char here[4096];
    if (in_dir(dir, here)) return -1;
    midfield(tstep, fileno, tval, outtime, outmid, cavgtime, g_grid, g_c, g_u, g_v, g_w);
    return chdir(here);
}

int pllref_intermediate(const char *dir, int *tstep, int *fileno, double *tval, double *outtime)
{
    char here[4096];
    if (in_dir(dir, here)) return -1;
    intermediate(tstep, fileno, tval, outtime, g_grid, g_c, g_u, g_v, g_w);
    return chdir(here);
}

int pllref_conc_average(double tval, const char *dir)
{
    char here[4096];
    if (in_dir(dir, here)) return -1;
    conc_average(g_grid, g_c->new, tval);
    return chdir(here);
}

int pllref_find_wmax(double tval, const char *dir)
{
    char here[4096];
    if (in_dir(dir, here)) return -1;
    find_wmax(tval, g_grid, g_w);
    return chdir(here);
}

int pllref_find_max(const char *dir)
{
    char here[4096];
    if (in_dir(dir, here)) return -1;
    find_max(g_grid, g_u, g_v, g_w, g_c);
    return chdir(here);
}

/* shift_conc (pllcart3d.c:3231) with the given wave parameters */
void pllref_shift_conc(double ampli, double lamb, int subharm)
{
    Ampli = ampli;
    Lamb = lamb;
    Subharm = subharm;
    shift_conc(g_grid, g_c);
}
