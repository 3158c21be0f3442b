/*
 * FFTW stand-in (see fftw3.h).  Test infrastructure only.
 */
#include "fftw3.h"
#include "../dct_def.h"

#include <stdio.h>
#include <stdlib.h>

struct pll_fftw_plan_s {
    int n0, n1, howmany, kind;
    long idist, odist;
    double *in, *out;
    double *T0, *T1, *tmp;
};

static int g_fast = 0;

void pll_shim_fftw_set_fast(int fast) { g_fast = fast; }

void *fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void *p) { free(p); }

fftw_plan fftw_plan_many_r2r(int rank, const int *n, int howmany, double *in,
                             const int *inembed, int istride, int idist,
                             double *out, const int *onembed, int ostride,
                             int odist, const fftw_r2r_kind *kind,
                             unsigned flags)
{
    fftw_plan p;
    int kk;
    (void)flags;
    if (rank != 2 || inembed || onembed || istride != 1 || ostride != 1 ||
        kind[0] != kind[1] ||
        (kind[0] != FFTW_REDFT10 && kind[0] != FFTW_REDFT01)) {
        fprintf(stderr, "fftw stand-in: unsupported plan\n");
        abort();
    }
    kk = (kind[0] == FFTW_REDFT10) ? PLL_DCT_II : PLL_DCT_III;
    p = (fftw_plan)calloc(1, sizeof(*p));
    p->n0 = n[0];
    p->n1 = n[1];
    p->howmany = howmany;
    p->kind = kk;
    p->idist = idist;
    p->odist = odist;
    p->in = in;
    p->out = out;
    p->T0 = (double *)malloc(sizeof(double) * (size_t)n[0] * n[0]);
    p->T1 = (double *)malloc(sizeof(double) * (size_t)n[1] * n[1]);
    p->tmp = (double *)malloc(sizeof(double) * (size_t)n[0] * n[1]);
    pll_dct_matrix(kk, n[0], p->T0);
    pll_dct_matrix(kk, n[1], p->T1);
    return p;
}

void fftw_execute(const fftw_plan p)
{
    int t;
    for (t = 0; t < p->howmany; t++) {
        const double *x = p->in + (long)t * p->idist;
        double *y = p->out + (long)t * p->odist;
        if (g_fast)
            pll_dct2d_fast(p->kind, p->n0, p->n1, x, y, p->tmp);
        else
            pll_dct2d_exact(p->kind, p->n0, p->n1, p->T0, p->T1, x, y, p->tmp);
    }
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    free(p->T0);
    free(p->T1);
    free(p->tmp);
    free(p);
}
