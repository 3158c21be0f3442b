/*
 * FFTW's published real-to-real cosine transforms, restated in plain C.
 * Test infrastructure only (oracle and the FFTW stand-in used to compile the
 * reference); never linked into the GPU library.
 *
 * The reference calls FFTW 3.2.2 (Makefile:35, pllcart3d.c:28) through
 * fftw_3d.h:12-106 with kinds REDFT10 (forward) and REDFT01 (inverse) on a
 * rank-2 transform of dims {nz, ny} (fftw_3d.h:23-24), batched over nx
 * planes.  FFTW is not vendored in the reference and not installed here, so
 * the transforms are restated from FFTW's documented definitions
 * (FFTW 3 manual, "1d Real-even DFTs (DCTs)"):
 *   REDFT10 (DCT-II):  Y_k = 2 sum_{j=0}^{n-1} X_j cos(pi (2j+1) k / (2n))
 *   REDFT01 (DCT-III): Y_k = X_0 + 2 sum_{j=1}^{n-1} X_j cos(pi j (2k+1) / (2n))
 * A multi-dimensional r2r transform is the separable product of the 1-d
 * transforms along each dimension (both unnormalised).
 */
#ifndef PLL_DCT_DEF_H
#define PLL_DCT_DEF_H

#ifdef __cplusplus
extern "C" {
#endif

enum { PLL_DCT_II = 0, PLL_DCT_III = 1 };

/* Dense transform matrix T[k*n + j] for one 1-d transform of length n. */
void pll_dct_matrix(int kind, int n, double *T);

/*
 * Exact-definition 2-d transform of one row-major n0 x n1 array (n1 fastest):
 * first along the fast dimension for every row, then along the slow
 * dimension for every column; each output is a sequential sum over the input
 * index in increasing order, acc = acc + T*x.  tmp holds n0*n1 doubles.
 */
void pll_dct2d_exact(int kind, int n0, int n1, const double *T0,
                     const double *T1, const double *in, double *out,
                     double *tmp);

/*
 * O(n log n) variant (Makhoul's reordering around a radix-2 complex FFT) for
 * power-of-two lengths; other lengths fall back to the dense sum.  Used only
 * to time the reference CPU path with a DCT as fast as FFTW's would be.
 */
void pll_dct2d_fast(int kind, int n0, int n1, const double *in, double *out,
                    double *tmp);

#ifdef __cplusplus
}
#endif
#endif
