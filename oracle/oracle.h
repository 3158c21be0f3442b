/*
 * CPU restatement of pllcart3d's RK3-CN time step (one MPI rank), written
 * by this project from the reference's algorithm.  TEST INFRASTRUCTURE ONLY:
 * the checker that the GPU library is compared against in tests/, in
 * __graft_entry__.smoke() and in the CPU-baseline leg of bench.py.  It is
 * never linked into, or called by, the GPU product.
 *
 * Fields are flat float64 arrays over the padded box (nx+6, ny+2, nz+2) with
 * z fastest: element (i,j,k) is at ((i*NY)+j)*NZ+k, the reference's
 * double***[i][j][k] order (allocate_3d_calloc.h:46-64).
 *
 * Parity: pinned bit-for-bit against the reference's own pllcart3d.c,
 * compiled by oracle/Makefile with single-rank MPI and FFTW stand-ins
 * (tests/test_oracle_pin.py); both sides use the same FFTW-definition DCT
 * (dct_def.c), so the pin covers every routine of the step.
 */
#ifndef PLL_ORACLE_H
#define PLL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

/*
 * dv: X1 X2 Y1 Y2 Z1 Z2 Re Pe Vratio Fx Fy CFLmax Timestep Mum Lambda
 * iv: Nx Ny Nz Nmvp
 */
orc *orc_create(const double *dv, const int *iv);
void orc_destroy(orc *o);
void orc_set_fast_dct(orc *o, int fast);
int orc_load_ic(orc *o, const double *c, const double *u, const double *v,
                const double *w);
int orc_steps(orc *o, int n);
void orc_substep(orc *o, double dt, int rk);
double orc_step_dt(orc *o);
double orc_last_dt(orc *o);
double orc_timestep(orc *o);
double orc_find_cfl(orc *o);
double orc_bulk_velo(orc *o);
double *orc_field(orc *o, const char *name);
int orc_call(orc *o, const char *routine, double a, double b, double c,
             double d);

/* stand-alone numerics */
double orc_weno(const double *d1, int kk, int sign);
void orc_thomas_serial(int n, const double *a, const double *b,
                       const double *c, double *r);
void orc_thomas_pll(int n, const double *a, double *b, double *c, double *r);

#ifdef __cplusplus
}
#endif
#endif
