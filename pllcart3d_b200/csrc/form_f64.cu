// The FP64 form of the step: FP64 state and arithmetic throughout, compiled
// with multiply-add contraction, the DCT passes of the Poisson solve as FFTs
// (power-of-two planes; the FP64 tensor-core contraction otherwise) and the
// WENO5 weights with one division.  It tracks the reference to rounding
// level; the exact form (form_f64x.cu) keeps the reference's operation
// order where a test needs bit-for-bit agreement.
#define PLL_FP64_EXACT 0
#include "orchestrate.cuh"

PLL_DEFINE_FORM(f64, double)
