// The precision form's FP32 kernels, compiled with multiply-add contraction
// (its accuracy contract is FP32-level, not the reference's op order).
#include "orchestrate.cuh"

PLL_DEFINE_FORM(f32, float)
