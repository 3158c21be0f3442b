// The plain FP64 form of the step: the reference's arithmetic, compiled
// without multiply-add contraction (--fmad=false).
#include "orchestrate.cuh"

PLL_DEFINE_FORM(f64, double)
