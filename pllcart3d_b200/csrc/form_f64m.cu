// The FP64-state form with FP32 WENO5 weights (PLLGPU_MIXED64): the FP64
// form's kernels and storage, except that each WENO5 derivative evaluates
// its smoothness indicators and nonlinear weights in FP32 from the FP64
// divided differences (the differences, the linear stencils of the
// diffusion and stress terms, the sums into the state and every solve stay
// FP64).  Compiled with multiply-add contraction.
#define PLL_FP64_EXACT 0
#define PLL_WENO_F32 1
#include "orchestrate.cuh"

PLL_DEFINE_FORM(f64m, double)
