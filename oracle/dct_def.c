/*
 * FFTW REDFT10 / REDFT01 restated from FFTW's documented definitions
 * (see dct_def.h).  Test infrastructure only.
 */
#include "dct_def.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double kPi = 3.14159265358979323846;

void pll_dct_matrix(int kind, int n, double *T)
{
    int k, j;
    for (k = 0; k < n; k++) {
        for (j = 0; j < n; j++) {
            long m;
            if (kind == PLL_DCT_II) {
                /* 2 cos(pi (2j+1) k / 2n), argument reduced mod 4n exactly */
                m = ((long)(2 * j + 1) * (long)k) % (4L * n);
                T[(long)k * n + j] = 2.0 * cos(kPi * (double)m / (2.0 * n));
            } else {
                if (j == 0) {
                    T[(long)k * n + j] = 1.0;
                } else {
                    m = ((long)j * (long)(2 * k + 1)) % (4L * n);
                    T[(long)k * n + j] = 2.0 * cos(kPi * (double)m / (2.0 * n));
                }
            }
        }
    }
}

void pll_dct2d_exact(int kind, int n0, int n1, const double *T0,
                     const double *T1, const double *in, double *out,
                     double *tmp)
{
    int r, c, k, j;
    (void)kind;
    /* along the fast dimension (length n1) for each of the n0 rows */
    for (r = 0; r < n0; r++) {
        const double *x = in + (long)r * n1;
        for (k = 0; k < n1; k++) {
            const double *t = T1 + (long)k * n1;
            double acc = 0.0;
            for (j = 0; j < n1; j++) acc = acc + t[j] * x[j];
            tmp[(long)r * n1 + k] = acc;
        }
    }
    /* along the slow dimension (length n0) for each of the n1 columns */
    for (c = 0; c < n1; c++) {
        for (k = 0; k < n0; k++) {
            const double *t = T0 + (long)k * n0;
            double acc = 0.0;
            for (j = 0; j < n0; j++) acc = acc + t[j] * tmp[(long)j * n1 + c];
            out[(long)k * n1 + c] = acc;
        }
    }
}

/* ---------------- fast variant (timing stand-in for FFTW) ---------------- */

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* in-place radix-2 complex FFT; sgn=-1 forward, +1 unnormalised inverse */
static void fft_radix2(int n, double *re, double *im, int sgn)
{
    int i, j, len;
    for (i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (len = 2; len <= n; len <<= 1) {
        double ang = sgn * 2.0 * kPi / len;
        int half = len >> 1, s, m;
        for (m = 0; m < half; m++) {
            double wr = cos(ang * m), wi = sin(ang * m);
            for (s = 0; s < n; s += len) {
                int a = s + m, b = s + m + half;
                double xr = re[b] * wr - im[b] * wi;
                double xi = re[b] * wi + im[b] * wr;
                re[b] = re[a] - xr; im[b] = im[a] - xi;
                re[a] += xr; im[a] += xi;
            }
        }
    }
}

/* one 1-d transform of length n with arbitrary strides */
static void dct1d_fast(int kind, int n, const double *x, long xs, double *y,
                       long ys, double *re, double *im)
{
    int k, j;
    if (kind == PLL_DCT_II) {
        for (j = 0; j < n / 2; j++) {
            re[j] = x[(long)(2 * j) * xs];
            re[n - 1 - j] = x[(long)(2 * j + 1) * xs];
        }
        memset(im, 0, sizeof(double) * (size_t)n);
        fft_radix2(n, re, im, -1);
        for (k = 0; k < n; k++) {
            double a = -kPi * k / (2.0 * n);
            y[(long)k * ys] = 2.0 * (cos(a) * re[k] - sin(a) * im[k]);
        }
    } else {
        for (k = 0; k < n; k++) {
            double xr = x[(long)k * xs];
            double xi = (k == 0) ? 0.0 : -x[(long)(n - k) * xs];
            double a = kPi * k / (2.0 * n);
            double c = cos(a), s = sin(a);
            re[k] = c * xr - s * xi;
            im[k] = s * xr + c * xi;
        }
        fft_radix2(n, re, im, +1);
        for (j = 0; j < n / 2; j++) {
            y[(long)(2 * j) * ys] = re[j];
            y[(long)(2 * j + 1) * ys] = re[n - 1 - j];
        }
    }
}

void pll_dct2d_fast(int kind, int n0, int n1, const double *in, double *out,
                    double *tmp)
{
    int r, c, nmax = n0 > n1 ? n0 : n1;
    double *re, *im;
    if (!is_pow2(n0) || !is_pow2(n1) || n0 < 2 || n1 < 2) {
        double *T0 = (double *)malloc(sizeof(double) * (size_t)n0 * n0);
        double *T1 = (double *)malloc(sizeof(double) * (size_t)n1 * n1);
        pll_dct_matrix(kind, n0, T0);
        pll_dct_matrix(kind, n1, T1);
        pll_dct2d_exact(kind, n0, n1, T0, T1, in, out, tmp);
        free(T0);
        free(T1);
        return;
    }
    re = (double *)malloc(sizeof(double) * (size_t)nmax);
    im = (double *)malloc(sizeof(double) * (size_t)nmax);
    for (r = 0; r < n0; r++)
        dct1d_fast(kind, n1, in + (long)r * n1, 1, tmp + (long)r * n1, 1, re, im);
    for (c = 0; c < n1; c++)
        dct1d_fast(kind, n0, tmp + c, n1, out + c, n1, re, im);
    free(re);
    free(im);
}
