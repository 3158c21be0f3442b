/*
 * CPU restatement of the pllcart3d RK3-CN step on one rank.
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the GPU library.
 *
 * Every routine names the reference lines it restates (pllcart3d.c unless
 * another file is named).  Arithmetic follows the reference expression by
 * expression, left to right, with no contracted multiply-adds, so that the
 * restatement reproduces the reference bit for bit; the structure (flat
 * arrays, one generic upwind pass, one generic implicit solve) is this
 * project's own.
 */
#include "oracle.h"
#include "dct_def.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int is, ie, js, je, ks, ke;
} rng3;

enum { VC = 0, VU = 1, VV = 2, VW = 3 };
enum { MU_CELL = 0, MU_XY = 1, MU_XZ = 2, MU_YZ = 3 };

struct orc {
    int nx, ny, nz;       /* interior cells */
    int NX, NY, NZ;       /* padded extents */
    long SX, SY;          /* strides of i and j */
    int nmax;             /* nmax_xyz, pllcart3d.c:372-373 */
    double dx, dy, dz;
    double X1, X2, Y1, Y2, Z1, Z2;
    double Re, Pe, M, Vnorm, Fx, Fy, CFLmax, Timestep, Mum, Lambda, PI;
    int nmvp, fast_dct;
    double cm;
    rng3 g, r[4];         /* grid range and per-variable unknown ranges */
    double *c_old, *c_new, *c_hn, *c_hnm1;
    double *q_old[4], *q_new[4], *q_hn[4], *q_hnm1[4], *q_pg[4];
    double *mu_old[4], *mu_new[4];
    double *phi, *div;
    /* scratch */
    double *src, *conv[3], *D1, *D2;
    double *la, *lb, *lc, *lr, *lw;
    double *Ty, *Tz, *Tiy, *Tiz, *plane_in, *plane_out, *plane_tmp;
    double *hat;
    double last_dt, tval;
};

#define AT(o, i, j, k) (((long)(i) * (o)->NY + (j)) * (o)->NZ + (k))

static const double RK1[3] = {(8.0 / 15.0), (5.0 / 12.0), (3.0 / 4.0)};
static const double RK2[3] = {(0.0), (-17.0 / 60.0), (-5.0 / 12.0)};

/* ------------------------------------------------------------------------ */
/* numerics kernels                                                          */
/* ------------------------------------------------------------------------ */

/* WENO5 derivative from five divided differences, pllcart3d.c:3455-3507 */
double orc_weno(const double *d1, int kk, int sign)
{
    const double con1 = 1.0 / 6.0, con2 = 13.0 / 12.0, con3 = 1.0 / 4.0;
    double v0 = d1[kk], v1 = d1[kk + sign], v2 = d1[kk + 2 * sign],
           v3 = d1[kk + 3 * sign], v4 = d1[kk + 4 * sign];
    double vs[5], maxd = 0.0, t1, t2, s1, s2, s3, c1, c2, c3, eps, a1, a2, a3,
                  at;
    int m;
    vs[0] = v0; vs[1] = v1; vs[2] = v2; vs[3] = v3; vs[4] = v4;
    for (m = 0; m < 5; m++) {
        double sq = vs[m] * vs[m];
        maxd = (maxd > sq) ? maxd : sq;
    }
    c1 = con1 * (2.0 * v0 - 7.0 * v1 + 11.0 * v2);
    c2 = con1 * (-1.0 * v1 + 5.0 * v2 + 2.0 * v3);
    c3 = con1 * (2.0 * v2 + 5.0 * v3 - 1.0 * v4);
    t1 = v0 - 2.0 * v1 + 1.0 * v2;
    t2 = v0 - 4.0 * v1 + 3.0 * v2;
    s1 = (con2 * t1 * t1) + (con3 * t2 * t2);
    t1 = v1 - 2.0 * v2 + v3;
    t2 = v1 - v3;
    s2 = (con2 * t1 * t1) + (con3 * t2 * t2);
    t1 = 1.0 * v2 - 2.0 * v3 + v4;
    t2 = 3.0 * v2 - 4.0 * v3 + v4;
    s3 = (con2 * t1 * t1) + (con3 * t2 * t2);
    eps = 1.0e-6 * maxd + 1.0e-99;
    a1 = 0.1 / ((s1 + eps) * (s1 + eps));
    a2 = 0.6 / ((s2 + eps) * (s2 + eps));
    a3 = 0.3 / ((s3 + eps) * (s3 + eps));
    at = a1 + a2 + a3;
    return (a1 / at) * c1 + (a2 / at) * c2 + (a3 / at) * c3;
}

/* Thomas solve without pivoting, tridiag_1rhs (pllcart3d.c:3511-3536).
 * Solution overwrites r; a, b, c untouched. */
void orc_thomas_serial(int n, const double *a, const double *b,
                       const double *c, double *r)
{
    double *cc = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double bb;
    int i;
    bb = b[0];
    cc[0] = c[0] / bb;
    r[0] = r[0] / bb;
    for (i = 1; i < n; i++) {
        bb = b[i] - cc[i - 1] * a[i];
        cc[i] = c[i] / bb;
        r[i] = (r[i] - r[i - 1] * a[i]) / bb;
    }
    for (i = n - 2; i >= 0; i--) r[i] = r[i] - r[i + 1] * cc[i];
    free(cc);
}

/* pll_tridiag on one rank (pll_tridiag.c:21-47, 96-110 with zero boundary
 * messages): b and c are overwritten with the eliminated coefficients. */
void orc_thomas_pll(int n, const double *a, double *b, double *c, double *r)
{
    int i;
    b[0] = b[0] - 0.0 * a[0];
    c[0] = c[0] / b[0];
    r[0] = (r[0] - 0.0 * a[0]) / b[0];
    for (i = 1; i < n; i++) {
        b[i] = (b[i] - c[i - 1] * a[i]);
        c[i] = c[i] / b[i];
        r[i] = (r[i] - r[i - 1] * a[i]) / b[i];
    }
    r[n - 1] = r[n - 1] - c[n - 1] * 0.0;
    for (i = n - 2; i >= 0; i--) r[i] = r[i] - c[i] * r[i + 1];
}

/* ------------------------------------------------------------------------ */
/* set-up                                                                    */
/* ------------------------------------------------------------------------ */

static double *zalloc(long n) { return (double *)calloc((size_t)n, sizeof(double)); }

orc *orc_create(const double *dv, const int *iv)
{
    orc *o = (orc *)calloc(1, sizeof(orc));
    long n;
    int v;
    o->X1 = dv[0]; o->X2 = dv[1]; o->Y1 = dv[2]; o->Y2 = dv[3];
    o->Z1 = dv[4]; o->Z2 = dv[5]; o->Re = dv[6]; o->Pe = dv[7];
    o->M = dv[8]; /* M = Vratio, pllcart3d.c:400 */
    o->Vnorm = 0.0; /* pllcart3d.c:403 */
    o->Fx = dv[9]; o->Fy = dv[10]; o->CFLmax = dv[11]; o->Timestep = dv[12];
    o->Mum = dv[13]; o->Lambda = dv[14];
    o->PI = 4.0 * atan(1.0);
    o->nx = iv[0]; o->ny = iv[1]; o->nz = iv[2]; o->nmvp = iv[3];
    if (o->nx < 4 || o->ny < 4 || o->nz < 4) { free(o); return NULL; }
    /* grid_setup, pllcart3d.c:357-382 (one rank, ghosts 3/1/1) */
    o->NX = o->nx + 6; o->NY = o->ny + 2; o->NZ = o->nz + 2;
    o->SY = o->NZ; o->SX = (long)o->NY * o->NZ;
    o->nmax = o->NX > o->NY ? o->NX : o->NY;
    o->nmax = o->nmax > o->NZ ? o->nmax : o->NZ;
    o->dx = (o->X2 - o->X1) / (double)o->nx;
    o->dy = (o->Y2 - o->Y1) / (double)o->ny;
    o->dz = (o->Z2 - o->Z1) / (double)o->nz;
    o->g.is = 3; o->g.ie = o->nx + 2;
    o->g.js = 1; o->g.je = o->ny;
    o->g.ks = 1; o->g.ke = o->nz;
    /* per-variable unknown ranges, simulation_setup pllcart3d.c:405-431 */
    for (v = 0; v < 4; v++) o->r[v] = o->g;
    o->r[VU].is = o->g.is + 1;  /* inlet face is fixed */
    o->r[VV].js = o->g.js + 1;  /* bottom wall face */
    o->r[VW].ks = o->g.ks + 1;  /* side wall face */

    n = (long)o->NX * o->SX;
    o->c_old = zalloc(n); o->c_new = zalloc(n);
    o->c_hn = zalloc(n); o->c_hnm1 = zalloc(n);
    for (v = 1; v < 4; v++) {
        o->q_old[v] = zalloc(n); o->q_new[v] = zalloc(n);
        o->q_hn[v] = zalloc(n); o->q_hnm1[v] = zalloc(n);
        o->q_pg[v] = zalloc(n);
    }
    o->q_old[0] = o->c_old; o->q_new[0] = o->c_new;
    o->q_hn[0] = o->c_hn; o->q_hnm1[0] = o->c_hnm1;
    for (v = 0; v < 4; v++) { o->mu_old[v] = zalloc(n); o->mu_new[v] = zalloc(n); }
    o->phi = zalloc(n); o->div = zalloc(n);
    o->src = zalloc(n);
    for (v = 0; v < 3; v++) o->conv[v] = zalloc(n);
    o->D1 = zalloc(o->nmax); o->D2 = zalloc(o->nmax);
    o->la = zalloc(o->nmax); o->lb = zalloc(o->nmax); o->lc = zalloc(o->nmax);
    o->lr = zalloc(o->nmax); o->lw = zalloc(o->nmax);
    o->Ty = zalloc((long)o->ny * o->ny); o->Tz = zalloc((long)o->nz * o->nz);
    o->Tiy = zalloc((long)o->ny * o->ny); o->Tiz = zalloc((long)o->nz * o->nz);
    pll_dct_matrix(PLL_DCT_II, o->ny, o->Ty);
    pll_dct_matrix(PLL_DCT_II, o->nz, o->Tz);
    pll_dct_matrix(PLL_DCT_III, o->ny, o->Tiy);
    pll_dct_matrix(PLL_DCT_III, o->nz, o->Tiz);
    o->plane_in = zalloc((long)o->ny * o->nz);
    o->plane_out = zalloc((long)o->ny * o->nz);
    o->plane_tmp = zalloc((long)o->ny * o->nz);
    o->hat = zalloc((long)o->nx * o->ny * o->nz);
    return o;
}

void orc_destroy(orc *o)
{
    int v;
    if (!o) return;
    free(o->c_old); free(o->c_new); free(o->c_hn); free(o->c_hnm1);
    for (v = 1; v < 4; v++) {
        free(o->q_old[v]); free(o->q_new[v]); free(o->q_hn[v]);
        free(o->q_hnm1[v]); free(o->q_pg[v]);
    }
    for (v = 0; v < 4; v++) { free(o->mu_old[v]); free(o->mu_new[v]); }
    free(o->phi); free(o->div); free(o->src);
    for (v = 0; v < 3; v++) free(o->conv[v]);
    free(o->D1); free(o->D2); free(o->la); free(o->lb); free(o->lc);
    free(o->lr); free(o->lw);
    free(o->Ty); free(o->Tz); free(o->Tiy); free(o->Tiz);
    free(o->plane_in); free(o->plane_out); free(o->plane_tmp); free(o->hat);
    free(o);
}

void orc_set_fast_dct(orc *o, int fast) { o->fast_dct = fast; }

double *orc_field(orc *o, const char *name)
{
    static const char *qn[4] = {"c", "u", "v", "w"};
    static const char *mn[4] = {"cell", "xy", "xz", "yz"};
    char buf[32];
    int v;
    for (v = 0; v < 4; v++) {
        strcpy(buf, qn[v]); strcat(buf, "_old");
        if (!strcmp(name, buf)) return o->q_old[v];
        strcpy(buf, qn[v]); strcat(buf, "_new");
        if (!strcmp(name, buf)) return o->q_new[v];
        strcpy(buf, qn[v]); strcat(buf, "_hn");
        if (!strcmp(name, buf)) return o->q_hn[v];
        strcpy(buf, qn[v]); strcat(buf, "_hnm1");
        if (!strcmp(name, buf)) return o->q_hnm1[v];
        strcpy(buf, qn[v]); strcat(buf, "_pg");
        if (v > 0 && !strcmp(name, buf)) return o->q_pg[v];
    }
    for (v = 0; v < 4; v++) {
        strcpy(buf, "mu_old_"); strcat(buf, mn[v]);
        if (!strcmp(name, buf)) return o->mu_old[v];
        strcpy(buf, "mu_new_"); strcat(buf, mn[v]);
        if (!strcmp(name, buf)) return o->mu_new[v];
    }
    if (!strcmp(name, "phi")) return o->phi;
    if (!strcmp(name, "div")) return o->div;
    return NULL;
}

/* ------------------------------------------------------------------------ */
/* viscosity, pllcart3d.c:843-886 (Nmvp=0) and 889-948 (Nmvp=1)             */
/* ------------------------------------------------------------------------ */

typedef struct {
    double mum, psi0, psi1, a;
} nmvp_coef;

static nmvp_coef nmvp_setup(const orc *o, double cm)
{
    nmvp_coef k;
    double alpha = exp(o->M), etam;
    k.mum = o->Mum * alpha;
    k.psi0 = asin(alpha / k.mum);
    k.psi1 = o->PI - asin(1 / k.mum);
    etam = (o->PI / 2 - k.psi0) / (k.psi1 - k.psi0);
    k.a = ((1 - cm) - etam) / ((1 - cm) * (etam - 1));
    return k;
}

static double visc_law(const orc *o, const nmvp_coef *k, double cavg)
{
    if (!o->nmvp) return exp(o->M * (cavg - o->Vnorm));
    {
        double eta = ((1 + k->a) * cavg) / (1 + k->a * cavg);
        double psi = k->psi1 * (1 - eta) + k->psi0 * eta;
        return k->mum * sin(psi);
    }
}

static void viscosity(orc *o, const double *cn, double *const mu[4])
{
    const rng3 *g = &o->g;
    nmvp_coef k;
    int i, j, kk;
    long SX = o->SX, SY = o->SY;
    memset(&k, 0, sizeof(k));
    if (o->nmvp) k = nmvp_setup(o, o->cm);
    for (i = g->is - 1; i <= g->ie + 1; i++)
        for (j = g->js - 1; j <= g->je + 1; j++)
            for (kk = g->ks - 1; kk <= g->ke + 1; kk++) {
                long id = AT(o, i, j, kk);
                mu[MU_CELL][id] = visc_law(o, &k, cn[id]);
            }
    for (i = g->is; i <= g->ie + 1; i++)
        for (j = g->js; j <= g->je + 1; j++)
            for (kk = g->ks; kk <= g->ke; kk++) {
                long id = AT(o, i, j, kk);
                double cavg = 0.25 * (cn[id - SX - SY] + cn[id - SY] +
                                      cn[id - SX] + cn[id]);
                mu[MU_XY][id] = visc_law(o, &k, cavg);
            }
    for (i = g->is; i <= g->ie + 1; i++)
        for (j = g->js; j <= g->je; j++)
            for (kk = g->ks; kk <= g->ke + 1; kk++) {
                long id = AT(o, i, j, kk);
                double cavg = 0.25 * (cn[id - SX - 1] + cn[id - 1] +
                                      cn[id - SX] + cn[id]);
                mu[MU_XZ][id] = visc_law(o, &k, cavg);
            }
    for (i = g->is; i <= g->ie; i++)
        for (j = g->js; j <= g->je + 1; j++)
            for (kk = g->ks; kk <= g->ke + 1; kk++) {
                long id = AT(o, i, j, kk);
                double cavg = 0.25 * (cn[id - SY - 1] + cn[id - 1] +
                                      cn[id - SY] + cn[id]);
                mu[MU_YZ][id] = visc_law(o, &k, cavg);
            }
}

/* slope_parameter, pllcart3d.c:722-840 (one rank); returns -1 when the
 * bisection does not converge within 500 iterations (the reference exits) */
static int slope_parameter(orc *o, const double *cn, double *cm_out)
{
    const rng3 *g = &o->g;
    int n = g->ie - g->is + 1, i, j, k, jj = g->js, kk = g->ks, idx1, idx2,
        niter = 0;
    double err, alpha, mum, psi0, psi1, etam, cL, cH, cm, errd, errl, a, eta,
        psi, mup1, mup2, lambda;
    double *croot = zalloc(n), *mucell = zalloc(n);
    err = 10.0;
    for (j = g->js; j <= g->je; j++) {
        double yc = o->Y1 - g->js * o->dy + (o->dy / 2.0) + j * o->dy;
        if (fabs(yc - 0.0) < err) { err = fabs(yc - 0.0); jj = j; }
    }
    err = 10.0;
    for (k = g->ks; k <= g->ke; k++) {
        double zc = o->Z1 - g->ks * o->dz + (o->dz / 2.0) + k * o->dz;
        if (fabs(zc - 0.0) < err) { err = fabs(zc - 0.0); kk = k; }
    }
    for (i = g->is; i <= g->ie; i++) croot[i - g->is] = cn[AT(o, i, jj, kk)];
    alpha = exp(o->M);
    mum = o->Mum * alpha;
    psi0 = asin(alpha / mum);
    psi1 = o->PI - asin(1 / mum);
    etam = (o->PI / 2 - psi0) / (psi1 - psi0);
    cL = 0.1; cH = 0.9;
    cm = 0.5 * (cL + cH);
    errd = 100; errl = 1e-5;
    while (errd > 1e-5) {
        a = ((1 - cm) - etam) / ((1 - cm) * (etam - 1));
        for (i = 0; i < n; i++) {
            eta = ((1 + a) * croot[i]) / (1 + a * croot[i]);
            psi = psi0 * (1 - eta) + psi1 * eta;
            mucell[i] = mum * sin(psi);
        }
        idx1 = -1;
        for (i = 0; i < n; i++) {
            if (idx1 > 0) break;
            if (fabs(croot[i]) > errl) idx1 = i;
        }
        idx2 = -1;
        for (i = n - 1; i >= 0; i--) {
            if (idx2 > 0) break;
            if (fabs(croot[i]) < 1 - errl) idx2 = i;
        }
        if (idx1 < 0 || idx2 < 1 || idx1 + 1 >= n) { free(croot); free(mucell); return -1; }
        mup1 = (mucell[idx1 + 1] - mucell[idx1]) / (croot[idx1 + 1] - croot[idx1]);
        mup2 = (mucell[idx2] - mucell[idx2 - 1]) / (croot[idx2] - croot[idx2 - 1]);
        lambda = (mup1 + mup2) / (alpha + 1);
        if (lambda > o->Lambda) cH = cm;
        else cL = cm;
        cm = 0.5 * (cL + cH);
        errd = fabs(lambda - o->Lambda);
        niter++;
        if (niter > 500) { free(croot); free(mucell); return -1; }
    }
    free(croot);
    free(mucell);
    *cm_out = cm;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* implicit-operator coefficients, pllcart3d.c:1411-1536                     */
/* ------------------------------------------------------------------------ */

static void acoef(const orc *o, int var, int axis, double *const mu[4], long id,
                  double *a, double *b, double *c)
{
    double del, h;
    switch (var) {
    case VC:
        h = axis == 0 ? o->dx : axis == 1 ? o->dy : o->dz;
        del = 1.0 / (o->Pe * h * h);
        *a = del;
        *c = del;
        break;
    case VU:
        if (axis == 0) {
            del = 2.0 / (o->Re * o->dx);
            *a = del * mu[MU_CELL][id - o->SX] / o->dx;
            *c = del * mu[MU_CELL][id] / o->dx;
        } else if (axis == 1) {
            del = 1.0 / (o->Re * o->dy);
            *a = del * mu[MU_XY][id] / o->dy;
            *c = del * mu[MU_XY][id + o->SY] / o->dy;
        } else {
            del = 1.0 / (o->Re * o->dz);
            *a = del * mu[MU_XZ][id] / o->dz;
            *c = del * mu[MU_XZ][id + 1] / o->dz;
        }
        break;
    case VV:
        if (axis == 0) {
            del = 1.0 / (o->Re * o->dx);
            *a = del * mu[MU_XY][id] / o->dx;
            *c = del * mu[MU_XY][id + o->SX] / o->dx;
        } else if (axis == 1) {
            del = 2.0 / (o->Re * o->dy);
            *a = del * mu[MU_CELL][id - o->SY] / o->dy;
            *c = del * mu[MU_CELL][id] / o->dy;
        } else {
            del = 1.0 / (o->Re * o->dz);
            *a = del * mu[MU_YZ][id] / o->dz;
            *c = del * mu[MU_YZ][id + 1] / o->dz;
        }
        break;
    default: /* VW */
        if (axis == 0) {
            del = 1.0 / (o->Re * o->dx);
            *a = del * mu[MU_XZ][id] / o->dx;
            *c = del * mu[MU_XZ][id + o->SX] / o->dx;
        } else if (axis == 1) {
            del = 1.0 / (o->Re * o->dy);
            *a = del * mu[MU_YZ][id] / o->dy;
            *c = del * mu[MU_YZ][id + o->SY] / o->dy;
        } else {
            del = 2.0 / (o->Re * o->dz);
            *a = del * mu[MU_CELL][id - 1] / o->dz;
            *c = del * mu[MU_CELL][id] / o->dz;
        }
        break;
    }
    *b = -(*a + *c);
}

/* ------------------------------------------------------------------------ */
/* explicit operators Hc/Hu/Hv/Hw, pllcart3d.c:1539-1980                     */
/* ------------------------------------------------------------------------ */

/* advecting velocity at point id of variable var for the pass along axis */
static double adv_vel(const orc *o, int var, int axis, double *const vel[4],
                      const double *self, long id)
{
    const double *un = vel[VU], *vn = vel[VV], *wn = vel[VW];
    long SX = o->SX, SY = o->SY;
    switch (var) {
    case VC: /* pllcart3d.c:1563, 1591, 1621 */
        if (axis == 0) return 0.5 * (un[id + SX] + un[id]);
        if (axis == 1) return 0.5 * (vn[id + SY] + vn[id]);
        return 0.5 * (wn[id + 1] + wn[id]);
    case VU: /* pllcart3d.c:1669, 1696, 1722 */
        if (axis == 0) return self[id];
        if (axis == 1)
            return 0.25 * (vn[id - SX] + vn[id] + vn[id + SY] + vn[id - SX + SY]);
        return 0.25 * (wn[id - SX] + wn[id] + wn[id + 1] + wn[id - SX + 1]);
    case VV: /* pllcart3d.c:1780, 1807, 1834 */
        if (axis == 0)
            return 0.25 * (un[id - SY] + un[id + SX - SY] + un[id] + un[id + SX]);
        if (axis == 1) return self[id];
        return 0.25 * (wn[id - SY] + wn[id - SY + 1] + wn[id] + wn[id + 1]);
    default: /* VW: pllcart3d.c:1892, 1919, 1946 */
        if (axis == 0)
            return 0.25 * (un[id - 1] + un[id + SX - 1] + un[id] + un[id + SX]);
        if (axis == 1)
            return 0.25 * (vn[id - 1] + vn[id] + vn[id + SY - 1] + vn[id + SY]);
        return self[id];
    }
}

/*
 * One directional upwind pass of an H*_op routine.  D1/D2 are the routine's
 * scratch lines: allocated zeroed once per routine call and reused by the x,
 * y and z passes in that order (e.g. pllcart3d.c:1545-1546).  Each pass
 * rewrites D1 on the whole padded line and D2 only on the variable's range,
 * so the ENO-2 closure's reads of D2 one point outside the range see what an
 * earlier pass left there - reproduced here by sharing D1/D2 the same way.
 * out[id] = (advecting velocity) * (upwind derivative).
 */
static void upwind_pass(orc *o, int var, int axis, const double *q,
                        double *const vel[4], double *out)
{
    const rng3 *r = &o->r[var];
    double *D1 = o->D1, *D2 = o->D2;
    double h = axis == 0 ? o->dx : axis == 1 ? o->dy : o->dz;
    long stride = axis == 0 ? o->SX : axis == 1 ? o->SY : 1;
    int npad = axis == 0 ? o->NX : axis == 1 ? o->NY : o->NZ;
    int s = axis == 0 ? r->is : axis == 1 ? r->js : r->ks;
    int e = axis == 0 ? r->ie : axis == 1 ? r->je : r->ke;
    /* the two outer loops in the reference's order */
    int o1s = axis == 0 ? r->js : r->is, o1e = axis == 0 ? r->je : r->ie;
    int o2s = axis == 2 ? r->js : r->ks, o2e = axis == 2 ? r->je : r->ke;
    int a1, a2, m;
    for (a1 = o1s; a1 <= o1e; a1++) {
        for (a2 = o2s; a2 <= o2e; a2++) {
            long base;
            if (axis == 0) base = AT(o, 0, a1, a2);
            else if (axis == 1) base = AT(o, a1, 0, a2);
            else base = AT(o, a1, a2, 0);
            for (m = 0; m < npad - 1; m++)
                D1[m] = (q[base + (m + 1) * stride] - q[base + m * stride]) / h;
            for (m = s; m <= e; m++) D2[m] = (D1[m] - D1[m - 1]) / (2.0 * h);
            for (m = s; m <= e; m++) {
                long id = base + m * stride;
                double vv = adv_vel(o, var, axis, vel, q, id), deriv;
                int sign = (vv >= 0.0) ? 1 : -1, kk;
                if ((m <= s + 1) | (m >= e - 1)) {
                    double d2val;
                    kk = (sign == 1) ? m - 1 : m;
                    d2val = (fabs(D2[kk]) <= fabs(D2[kk + 1])) ? D2[kk] : D2[kk + 1];
                    deriv = D1[kk] + d2val * h * sign;
                } else {
                    kk = m - 3 - (int)(2.5 * (sign - 1));
                    deriv = orc_weno(D1, kk, sign);
                }
                out[id] = vv * deriv;
            }
        }
    }
}

/* explicit operator of variable var into q_hn[var] (interior range) */
static void explicit_op(orc *o, int var, double *const vel[4],
                        double *const mu[4])
{
    const rng3 *r = &o->r[var];
    const double *q = o->q_old[var];
    double *H = o->q_hn[var];
    double *cx = o->conv[0], *cy = o->conv[1], *cz = o->conv[2];
    long SX = o->SX, SY = o->SY;
    int i, j, k;
    memset(o->D1, 0, sizeof(double) * o->nmax);
    memset(o->D2, 0, sizeof(double) * o->nmax);
    upwind_pass(o, var, 0, q, vel, cx);
    upwind_pass(o, var, 1, q, vel, cy);
    upwind_pass(o, var, 2, q, vel, cz);
    for (i = r->is; i <= r->ie; i++)
        for (j = r->js; j <= r->je; j++)
            for (k = r->ks; k <= r->ke; k++) {
                long id = AT(o, i, j, k);
                double ct = cz[id] + cx[id] + cy[id], del, s1, s2, s3, s4;
                const double *un = vel[VU], *vn = vel[VV], *wn = vel[VW];
                if (var == VC) { /* pllcart3d.c:1634 */
                    H[id] = -(ct);
                    continue;
                }
                if (var == VU) { /* pllcart3d.c:1736-1744 */
                    del = 1.0 / (o->Re * o->dy * o->dx);
                    s1 = del * mu[MU_XY][id + SY] * (vn[id + SY] - vn[id - SX + SY]);
                    s2 = del * mu[MU_XY][id] * (vn[id] - vn[id - SX]);
                    del = 1.0 / (o->Re * o->dz * o->dx);
                    s3 = del * mu[MU_XZ][id + 1] * (wn[id + 1] - wn[id - SX + 1]);
                    s4 = del * mu[MU_XZ][id] * (wn[id] - wn[id - SX]);
                } else if (var == VV) { /* pllcart3d.c:1848-1856 */
                    del = 1.0 / (o->Re * o->dx * o->dy);
                    s1 = del * mu[MU_XY][id + SX] * (un[id + SX] - un[id + SX - SY]);
                    s2 = del * mu[MU_XY][id] * (un[id] - un[id - SY]);
                    del = 1.0 / (o->Re * o->dz * o->dy);
                    s3 = del * mu[MU_YZ][id + 1] * (wn[id + 1] - wn[id - SY + 1]);
                    s4 = del * mu[MU_YZ][id] * (wn[id] - wn[id - SY]);
                } else { /* VW, pllcart3d.c:1960-1970 (index choice of L1962) */
                    del = 1.0 / (o->Re * o->dx * o->dz);
                    s1 = del * mu[MU_XZ][id + SX] * (un[id + SX] - un[id + SX - 1]);
                    s2 = del * mu[MU_XZ][id] * (un[id] - un[id - 1]);
                    del = 1.0 / (o->Re * o->dy * o->dz);
                    s3 = del * mu[MU_YZ][id + SY] * (vn[id + SY] - vn[id + SY - 1]);
                    s4 = del * mu[MU_YZ][id] * (vn[id] - vn[id - 1]);
                }
                H[id] = -ct + s1 - s2 + s3 - s4;
            }
}

/* ------------------------------------------------------------------------ */
/* implicit (ADI) update of one variable                                     */
/* concentration L573-712, xmom L970-1102, ymom L1127-1255, zmom L1280-1403  */
/* ------------------------------------------------------------------------ */

/* boundary closures; codes: 0 none, 1 b+=a (Neumann/symmetric),
 * 2 b-=a (reflection about a wall face), 3 rhs-=a*0 (Dirichlet face) */
static const int closure_lo[4][3] = {
    /* x: left, y: bottom, z: side (first unknown of each line) */
    {3, 1, 1}, /* c: L675, L610, L640 */
    {3, 2, 1}, /* u: L1075, L1010, L1039 */
    {2, 3, 1}, /* v: L1231, L1167, L1196 */
    {2, 2, 3}, /* w: L1378, L1317, L1344 */
};
static const int closure_hi[4][3] = {
    /* x: outflow handled separately (code 0 here), y: top, z: side */
    {0, 1, 1}, /* c: L611, L641 */
    {0, 2, 1}, /* u: L1011, L1040 */
    {0, 3, 1}, /* v: L1168, L1197 */
    {0, 2, 3}, /* w: L1318, L1345 */
};

static void apply_lo(int code, double *la, double *lb, double *lr)
{
    if (code == 1) lb[0] += la[0];
    else if (code == 2) lb[0] -= la[0];
    else if (code == 3) lr[0] -= la[0] * 0.0;
}

static void apply_hi(int code, int n, double *lb, double *lc, double *lr)
{
    if (code == 1) lb[n - 1] += lc[n - 1];
    else if (code == 2) lb[n - 1] -= lc[n - 1];
    else if (code == 3) lr[n - 1] -= lc[n - 1] * 0.0;
}

static void implicit_update(orc *o, int var, double dt, double g, double rr,
                            double vbulk, const double *cn,
                            double *const mu_o[4], double *const mu_n[4])
{
    const rng3 *r = &o->r[var];
    const double *q = o->q_old[var];
    double *qn = o->q_new[var], *H = o->q_hn[var], *Hm = o->q_hnm1[var];
    double *S = o->src;
    double alpha = g + rr, fac;
    long SX = o->SX, SY = o->SY;
    int i, j, k, m, n, axis;

    /* right-hand side */
    for (i = r->is; i <= r->ie; i++)
        for (j = r->js; j <= r->je; j++)
            for (k = r->ks; k <= r->ke; k++) {
                long id = AT(o, i, j, k);
                double a, b, c, ax, ay, az, conv, diff, bf, cval;
                conv = (g * H[id] + rr * Hm[id]);
                acoef(o, var, 0, mu_o, id, &a, &b, &c);
                ax = a * q[id - SX] + b * q[id] + c * q[id + SX];
                acoef(o, var, 1, mu_o, id, &a, &b, &c);
                ay = a * q[id - SY] + b * q[id] + c * q[id + SY];
                acoef(o, var, 2, mu_o, id, &a, &b, &c);
                az = a * q[id - 1] + b * q[id] + c * q[id + 1];
                diff = alpha * (ax + ay + az);
                if (var == VC) {
                    S[id] = dt * (conv + diff);
                } else {
                    if (var == VU) {
                        cval = 0.5 * (cn[id] + cn[id - SX]);
                        bf = alpha * (-(o->Fx / o->Re) * cval - (o->q_pg[var][id] / o->Re));
                    } else if (var == VV) {
                        cval = 0.5 * (cn[id] + cn[id - SY]);
                        bf = alpha * (-(o->Fy / o->Re) * cval - (o->q_pg[var][id] / o->Re));
                    } else {
                        bf = alpha * (-(o->q_pg[var][id] / o->Re));
                    }
                    S[id] = dt * (conv + diff + bf);
                }
            }

    fac = 0.5 * dt * alpha;

    /* y then z sweeps, serial Thomas (tridiag_1rhs) */
    for (axis = 1; axis <= 2; axis++) {
        long stride = axis == 1 ? SY : 1;
        int s = axis == 1 ? r->js : r->ks, e = axis == 1 ? r->je : r->ke;
        int o2s = axis == 1 ? r->ks : r->js, o2e = axis == 1 ? r->ke : r->je;
        n = e - s + 1;
        for (i = r->is; i <= r->ie; i++)
            for (j = o2s; j <= o2e; j++) {
                long base = axis == 1 ? AT(o, i, s, j) : AT(o, i, j, s);
                for (m = 0; m < n; m++) {
                    long id = base + m * stride;
                    double a, b, c;
                    acoef(o, var, axis, mu_n, id, &a, &b, &c);
                    o->la[m] = -fac * a;
                    o->lb[m] = 1.0 - fac * b;
                    o->lc[m] = -fac * c;
                    o->lr[m] = S[id];
                }
                apply_lo(closure_lo[var][axis], o->la, o->lb, o->lr);
                apply_hi(closure_hi[var][axis], n, o->lb, o->lc, o->lr);
                orc_thomas_serial(n, o->la, o->lb, o->lc, o->lr);
                for (m = 0; m < n; m++) S[base + m * stride] = o->lr[m];
            }
    }

    /* x sweep, pll_tridiag on one rank, with the outflow closure */
    n = r->ie - r->is + 1;
    for (j = r->js; j <= r->je; j++)
        for (k = r->ks; k <= r->ke; k++) {
            long base = AT(o, r->is, j, k), rb = AT(o, r->ie + 1, j, k);
            double boun;
            for (m = 0; m < n; m++) {
                long id = base + m * SX;
                double a, b, c;
                acoef(o, var, 0, mu_n, id, &a, &b, &c);
                o->la[m] = -fac * a;
                o->lb[m] = 1.0 - fac * b;
                o->lc[m] = -fac * c;
                o->lr[m] = S[id];
            }
            apply_lo(closure_lo[var][0], o->la, o->lb, o->lr);
            /* convective outflow, e.g. pllcart3d.c:677-683 */
            H[rb] = -vbulk * (q[rb] - q[rb - SX]) / o->dx;
            boun = dt * (g * H[rb] + rr * Hm[rb]);
            qn[rb] = q[rb] + boun;
            o->lr[n - 1] -= o->lc[n - 1] * boun;
            orc_thomas_pll(n, o->la, o->lb, o->lc, o->lr);
            for (m = 0; m < n; m++) {
                long id = base + m * SX;
                qn[id] = q[id] + o->lr[m];
            }
        }

    if (var == VC) { /* Neumann ghosts, pllcart3d.c:700-712 */
        for (i = r->is; i <= r->ie; i++)
            for (k = r->ks; k <= r->ke; k++) {
                qn[AT(o, i, r->js - 1, k)] = qn[AT(o, i, r->js, k)];
                qn[AT(o, i, r->je + 1, k)] = qn[AT(o, i, r->je, k)];
            }
        for (i = r->is; i <= r->ie; i++)
            for (j = r->js - 1; j <= r->je + 1; j++) {
                qn[AT(o, i, j, r->ks - 1)] = qn[AT(o, i, j, r->ks)];
                qn[AT(o, i, j, r->ke + 1)] = qn[AT(o, i, j, r->ke)];
            }
    }
}

/* ------------------------------------------------------------------------ */
/* step routines                                                             */
/* ------------------------------------------------------------------------ */

/* concentration, pllcart3d.c:555-719 */
static void concentration(orc *o, double dt, double g, double r, double vb)
{
    double *vel[4];
    vel[0] = NULL; vel[VU] = o->q_new[VU]; vel[VV] = o->q_new[VV]; vel[VW] = o->q_new[VW];
    explicit_op(o, VC, vel, NULL);
    implicit_update(o, VC, dt, g, r, vb, NULL, NULL, NULL);
}

/* xmom / ymom / zmom, pllcart3d.c:952-1408: the explicit operator sees the
 * *old* velocities of the other two components and mu_old; the implicit
 * coefficients are rebuilt from mu_new (L991, L1148, L1300) */
static void momentum(orc *o, int var, double dt, double g, double r, double vb)
{
    double *vel[4];
    vel[0] = NULL; vel[VU] = o->q_old[VU]; vel[VV] = o->q_old[VV]; vel[VW] = o->q_old[VW];
    explicit_op(o, var, vel, o->mu_old);
    implicit_update(o, var, dt, g, r, vb, o->c_new, o->mu_old, o->mu_new);
}

/* update_velo_boundary L2701-2755 and update_veloghost_points L2810-2885
 * (identical on one rank; exchanges are no-ops) */
static void velo_ghosts(orc *o)
{
    const rng3 *g = &o->g;
    double *u = o->q_new[VU], *v = o->q_new[VV], *w = o->q_new[VW];
    int i, j, k;
    for (i = g->is; i <= g->ie; i++)
        for (j = g->js; j <= g->je; j++) {
            u[AT(o, i, j, g->ks - 1)] = u[AT(o, i, j, g->ks)];
            v[AT(o, i, j, g->ks - 1)] = v[AT(o, i, j, g->ks)];
            u[AT(o, i, j, g->ke + 1)] = u[AT(o, i, j, g->ke)];
            v[AT(o, i, j, g->ke + 1)] = v[AT(o, i, j, g->ke)];
        }
    for (i = g->is; i <= g->ie; i++)
        for (k = g->ks; k <= g->ke; k++) {
            u[AT(o, i, g->js - 1, k)] = -u[AT(o, i, g->js, k)];
            w[AT(o, i, g->js - 1, k)] = -w[AT(o, i, g->js, k)];
            u[AT(o, i, g->je + 1, k)] = -u[AT(o, i, g->je, k)];
            w[AT(o, i, g->je + 1, k)] = -w[AT(o, i, g->je, k)];
        }
    for (j = g->js; j <= g->je; j++)
        for (k = g->ks; k <= g->ke; k++) {
            v[AT(o, g->is - 1, j, k)] = -v[AT(o, g->is, j, k)];
            w[AT(o, g->is - 1, j, k)] = -w[AT(o, g->is, j, k)];
        }
}

/* divergence, pllcart3d.c:1983-1999 */
static void divergence(orc *o)
{
    const rng3 *g = &o->g;
    const double *u = o->q_new[VU], *v = o->q_new[VV], *w = o->q_new[VW];
    int i, j, k;
    for (i = g->is; i <= g->ie; i++)
        for (j = g->js; j <= g->je; j++)
            for (k = g->ks; k <= g->ke; k++) {
                long id = AT(o, i, j, k);
                double dvx = (u[id + o->SX] - u[id]) / o->dx;
                double dvy = (v[id + o->SY] - v[id]) / o->dy;
                double dvz = (w[id + 1] - w[id]) / o->dz;
                o->div[id] = (dvx + dvy + dvz);
            }
}

/* phisolver_dct, pllcart3d.c:2002-2130 with fftw_3d.h:45-106:
 * per x-plane 2-d DCT-II over (z,y), an x-tridiagonal per (ky,kz) mode with
 * Neumann ends and the (0,0)-mode gauge phi=0 in the right ghost, then the
 * 2-d DCT-III divided by 4*ny*nz */
static void phisolver(orc *o, double dt, double g, double r)
{
    const rng3 *gr = &o->g;
    int nx = o->nx, ny = o->ny, nz = o->nz, i, j, k;
    long N = (long)ny * nz;
    double fac = o->Re / (dt * (g + r)), dx2i, phiconst = 0.0;
    double *hat = o->hat;
    for (i = 0; i < nx; i++) {
        /* plane layout [z][y], y fastest (fftw_3d.h:58) */
        for (j = 0; j < ny; j++)
            for (k = 0; k < nz; k++)
                o->plane_in[(long)k * ny + j] =
                    fac * o->div[AT(o, i + gr->is, j + gr->js, k + gr->ks)];
        if (o->fast_dct)
            pll_dct2d_fast(PLL_DCT_II, nz, ny, o->plane_in, hat + i * N, o->plane_tmp);
        else
            pll_dct2d_exact(PLL_DCT_II, nz, ny, o->Tz, o->Ty, o->plane_in,
                            hat + i * N, o->plane_tmp);
    }
    dx2i = 1.0 / (o->dx * o->dx);
    for (j = 0; j < ny; j++)
        for (k = 0; k < nz; k++) {
            double ki = 2.0 * (cos(o->PI * (double)j / (double)ny) - 1.0) / (o->dy * o->dy);
            double kk = 2.0 * (cos(o->PI * (double)k / (double)nz) - 1.0) / (o->dz * o->dz);
            for (i = 0; i < nx; i++) {
                o->la[i] = dx2i;
                o->lb[i] = -2.0 * dx2i + ki + kk;
                o->lc[i] = dx2i;
                o->lr[i] = hat[i * N + (long)k * ny + j];
            }
            o->lb[0] += o->la[0];
            if ((j == 0) && (k == 0)) o->lr[nx - 1] -= o->lc[nx - 1] * phiconst;
            else o->lb[nx - 1] += o->lc[nx - 1];
            orc_thomas_pll(nx, o->la, o->lb, o->lc, o->lr);
            for (i = 0; i < nx; i++) hat[i * N + (long)k * ny + j] = o->lr[i];
        }
    for (i = 0; i < nx; i++) {
        if (o->fast_dct)
            pll_dct2d_fast(PLL_DCT_III, nz, ny, hat + i * N, o->plane_out, o->plane_tmp);
        else
            pll_dct2d_exact(PLL_DCT_III, nz, ny, o->Tiz, o->Tiy, hat + i * N,
                            o->plane_out, o->plane_tmp);
        for (j = 0; j < ny; j++)
            for (k = 0; k < nz; k++)
                o->phi[AT(o, i + gr->is, j + gr->js, k + gr->ks)] =
                    o->plane_out[(long)k * ny + j] / (double)(4 * N);
    }
}

/* update_phi_ghosts, pllcart3d.c:2758-2807 */
static void phi_ghosts(orc *o)
{
    const rng3 *g = &o->g;
    double *p = o->phi;
    int i, j, k;
    for (i = g->is; i <= g->ie; i++)
        for (j = g->js; j <= g->je; j++) {
            p[AT(o, i, j, g->ks - 1)] = p[AT(o, i, j, g->ks)];
            p[AT(o, i, j, g->ke + 1)] = p[AT(o, i, j, g->ke)];
        }
    for (i = g->is; i <= g->ie; i++)
        for (k = g->ks; k <= g->ke; k++) {
            p[AT(o, i, g->js - 1, k)] = p[AT(o, i, g->js, k)];
            p[AT(o, i, g->je + 1, k)] = p[AT(o, i, g->je, k)];
        }
    for (j = g->js; j <= g->je; j++)
        for (k = g->ks; k <= g->ke; k++) {
            p[AT(o, g->is - 1, j, k)] = p[AT(o, g->is, j, k)];
            p[AT(o, g->ie + 1, j, k)] = p[AT(o, g->ie, j, k)];
        }
}

/* trapezoid flux through u-face plane i (z first, then y; wall half-cells
 * excluded), pllcart3d.c:2174-2185 and 2199-2210 */
static double face_flux(orc *o, int i)
{
    const rng3 *r = &o->r[VU];
    const double *u = o->q_new[VU];
    double *qk = o->lw, q;
    int j, k;
    for (j = r->js; j <= r->je; j++) {
        q = 0.0;
        for (k = r->ks + 1; k <= r->ke; k++)
            q += 0.5 * o->dz * (u[AT(o, i, j, k)] + u[AT(o, i, j, k - 1)]);
        qk[j] = q;
    }
    q = 0.0;
    for (j = r->js + 1; j <= r->je; j++) q += 0.5 * o->dy * (qk[j - 1] + qk[j]);
    return q;
}

/* velo_correction, pllcart3d.c:2133-2227 */
static void velo_correction(orc *o, double dt, double g, double r)
{
    double fac = dt * (g + r) / o->Re, qin, qout, deficit;
    int order[3] = {VV, VW, VU}, t, i, j, k;
    for (t = 0; t < 3; t++) {
        int v = order[t];
        const rng3 *rg = &o->r[v];
        long st = v == VU ? o->SX : v == VV ? o->SY : 1;
        double h = v == VU ? o->dx : v == VV ? o->dy : o->dz;
        double *q = o->q_new[v];
        for (i = rg->is; i <= rg->ie; i++)
            for (j = rg->js; j <= rg->je; j++)
                for (k = rg->ks; k <= rg->ke; k++) {
                    long id = AT(o, i, j, k);
                    double dphi = (o->phi[id] - o->phi[id - st]) / h;
                    q[id] = q[id] - fac * dphi;
                }
    }
    qin = face_flux(o, o->r[VU].is - 1);
    qout = face_flux(o, o->r[VU].ie + 1);
    deficit = (qin - qout) / ((o->Y2 - o->Y1) * (o->Z2 - o->Z1));
    for (j = o->r[VU].js; j <= o->r[VU].je; j++)
        for (k = o->r[VU].ks; k <= o->r[VU].ke; k++) {
            long id = AT(o, o->r[VU].ie + 1, j, k);
            o->q_new[VU][id] = o->q_new[VU][id] + deficit;
        }
}

/* pressure_gradient, pllcart3d.c:2964-3044: pg += grad(phi) - fac*A grad(phi)
 * with A built from mu_new; grad(phi) exists one point beyond the range */
static void pressure_gradient(orc *o, double dt, double g, double r)
{
    double fac = 0.5 * dt * (g + r);
    int order[3] = {VV, VU, VW}, t, i, j, k;
    for (t = 0; t < 3; t++) {
        int v = order[t];
        const rng3 *rg = &o->r[v];
        long st = v == VU ? o->SX : v == VV ? o->SY : 1;
        double h = v == VU ? o->dx : v == VV ? o->dy : o->dz;
        double *pg = o->q_pg[v], *gp = o->src;
        for (i = rg->is - 1; i <= rg->ie + 1; i++)
            for (j = rg->js - 1; j <= rg->je + 1; j++)
                for (k = rg->ks - 1; k <= rg->ke + 1; k++) {
                    long id = AT(o, i, j, k);
                    gp[id] = (o->phi[id] - o->phi[id - st]) / h;
                }
        for (i = rg->is; i <= rg->ie; i++)
            for (j = rg->js; j <= rg->je; j++)
                for (k = rg->ks; k <= rg->ke; k++) {
                    long id = AT(o, i, j, k);
                    double a, b, c, pxx, pyy, pzz;
                    acoef(o, v, 0, o->mu_new, id, &a, &b, &c);
                    pxx = a * gp[id - o->SX] + b * gp[id] + c * gp[id + o->SX];
                    acoef(o, v, 1, o->mu_new, id, &a, &b, &c);
                    pyy = a * gp[id - o->SY] + b * gp[id] + c * gp[id + o->SY];
                    acoef(o, v, 2, o->mu_new, id, &a, &b, &c);
                    pzz = a * gp[id - 1] + b * gp[id] + c * gp[id + 1];
                    pg[id] = pg[id] + gp[id] - fac * (pyy + pxx + pzz);
                }
    }
}

/* update_old_conc / update_old_velo / update_old_visc, L3402-3452 */
static void rotate(orc *o)
{
    long n = (long)o->NX * o->SX;
    int v;
    for (v = 0; v < 4; v++) {
        memcpy(o->q_old[v], o->q_new[v], sizeof(double) * n);
        memcpy(o->q_hnm1[v], o->q_hn[v], sizeof(double) * n);
        memcpy(o->mu_old[v], o->mu_new[v], sizeof(double) * n);
    }
}

/* find_cfl, pllcart3d.c:3095-3118 */
double orc_find_cfl(orc *o)
{
    const rng3 *g = &o->g;
    const double *u = o->q_old[VU], *v = o->q_old[VV], *w = o->q_old[VW];
    double maxval = 0.0;
    int i, j, k;
    for (i = g->is; i <= g->ie; i++)
        for (j = g->js; j <= g->je; j++)
            for (k = g->ks; k <= g->ke; k++) {
                long id = AT(o, i, j, k);
                double uv = 0.5 * (u[id] + u[id + o->SX]);
                double vv = 0.5 * (v[id] + v[id + o->SY]);
                double wv = 0.5 * (w[id] + w[id + 1]);
                double cfl = (fabs(uv) / o->dx) + (fabs(vv) / o->dy) + (fabs(wv) / o->dz);
                maxval = (cfl > maxval) ? cfl : maxval;
            }
    return o->CFLmax / maxval;
}

/* bulk_velo, pllcart3d.c:3381-3398: signed value of the first largest |u|
 * on the last interior u face */
double orc_bulk_velo(orc *o)
{
    const rng3 *g = &o->g;
    const double *u = o->q_old[VU];
    double vb = 0.0;
    int j, k;
    for (j = g->js; j <= g->je; j++)
        for (k = g->ks; k <= g->ke; k++) {
            double x = u[AT(o, g->ie, j, k)];
            if (fabs(x) > fabs(vb)) vb = x;
        }
    return vb;
}

double orc_step_dt(orc *o)
{
    double cfl_dt = orc_find_cfl(o);
    return (cfl_dt < o->Timestep) ? cfl_dt : o->Timestep;
}

/* one RK3-CN substep, pllcart3d.c:164-194 */
void orc_substep(orc *o, double dt, int rk)
{
    double g = RK1[rk], r = RK2[rk], vb;
    o->tval = o->tval + (g + r) * dt;
    vb = orc_bulk_velo(o);
    concentration(o, dt, g, r, vb);
    viscosity(o, o->c_new, o->mu_new);
    momentum(o, VU, dt, g, r, vb);
    momentum(o, VV, dt, g, r, vb);
    momentum(o, VW, dt, g, r, vb);
    velo_ghosts(o);
    divergence(o);
    phisolver(o, dt, g, r);
    phi_ghosts(o);
    velo_correction(o, dt, g, r);
    velo_ghosts(o);
    pressure_gradient(o, dt, g, r);
    rotate(o);
}

int orc_steps(orc *o, int n)
{
    int s, rk;
    for (s = 0; s < n; s++) {
        o->last_dt = orc_step_dt(o);
        for (rk = 0; rk < 3; rk++) orc_substep(o, o->last_dt, rk);
    }
    return 0;
}

double orc_last_dt(orc *o) { return o->last_dt; }
double orc_timestep(orc *o) { return o->Timestep; }

/* start-up after the initial fields, pllcart3d.c:81-83 and 126-154:
 * ghost fill of the initial velocities (update_ghost_points L2887-2961 with
 * phi = 0), new -> old, viscosity from c_old, diffusive cap of Timestep */
int orc_load_ic(orc *o, const double *c, const double *u, const double *v,
                const double *w)
{
    long n = (long)o->NX * o->SX;
    double dmin, diff_dt;
    memcpy(o->c_new, c, sizeof(double) * n);
    memcpy(o->q_new[VU], u, sizeof(double) * n);
    memcpy(o->q_new[VV], v, sizeof(double) * n);
    memcpy(o->q_new[VW], w, sizeof(double) * n);
    velo_ghosts(o);
    phi_ghosts(o); /* phi is zero: fills zeros */
    {
        int vv;
        for (vv = 0; vv < 4; vv++) {
            memcpy(o->q_old[vv], o->q_new[vv], sizeof(double) * n);
            memcpy(o->q_hnm1[vv], o->q_hn[vv], sizeof(double) * n);
        }
    }
    if (o->nmvp) {
        if (slope_parameter(o, o->c_new, &o->cm) != 0) return -1;
    }
    viscosity(o, o->c_old, o->mu_old);
    dmin = (o->dx < o->dy) ? o->dx : o->dy;
    dmin = (dmin < o->dz) ? dmin : o->dz;
    diff_dt = 0.1 * o->Pe * dmin * dmin;
    o->Timestep = (diff_dt < o->Timestep) ? diff_dt : o->Timestep;
    o->tval = 0.0;
    return 0;
}

/* single routines for per-routine parity; a..d are the routine's scalars */
int orc_call(orc *o, const char *routine, double a, double b, double c,
             double d)
{
    if (!strcmp(routine, "concentration")) concentration(o, a, b, c, d);
    else if (!strcmp(routine, "viscosity_new")) viscosity(o, o->c_new, o->mu_new);
    else if (!strcmp(routine, "xmom")) momentum(o, VU, a, b, c, d);
    else if (!strcmp(routine, "ymom")) momentum(o, VV, a, b, c, d);
    else if (!strcmp(routine, "zmom")) momentum(o, VW, a, b, c, d);
    else if (!strcmp(routine, "velo_ghosts")) velo_ghosts(o);
    else if (!strcmp(routine, "divergence")) divergence(o);
    else if (!strcmp(routine, "phisolver")) phisolver(o, a, b, c);
    else if (!strcmp(routine, "phi_ghosts")) phi_ghosts(o);
    else if (!strcmp(routine, "velo_correction")) velo_correction(o, a, b, c);
    else if (!strcmp(routine, "pressure_gradient")) pressure_gradient(o, a, b, c);
    else if (!strcmp(routine, "rotate")) rotate(o);
    else return -1;
    return 0;
}
