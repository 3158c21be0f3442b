/*
 * Stand-in for the subset of the FFTW 3 API that fftw_3d.h:12-106 of the
 * reference uses: fftw_plan_many_r2r (rank 2, contiguous, no embedding),
 * fftw_execute, fftw_malloc/fftw_free, kinds REDFT10/REDFT01.  Test
 * infrastructure only.  The transforms follow FFTW's documented definitions
 * (oracle/dct_def.h); FFTW itself is not installed in this image.
 * Names and enum values follow FFTW's public fftw3.h interface.
 */
#ifndef PLL_SHIM_FFTW3_H
#define PLL_SHIM_FFTW3_H

#include <stddef.h>

typedef enum {
    FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
    FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
    FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
} fftw_r2r_kind;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

typedef struct pll_fftw_plan_s *fftw_plan;

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_many_r2r(int rank, const int *n, int howmany, double *in,
                             const int *inembed, int istride, int idist,
                             double *out, const int *onembed, int ostride,
                             int odist, const fftw_r2r_kind *kind,
                             unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

/* stand-in control: 0 = dense exact-definition sums (default), 1 = FFT-based */
void pll_shim_fftw_set_fast(int fast);

#endif
