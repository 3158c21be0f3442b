// The precision form's FP32 kernels (its accuracy contract is FP32-level,
// not the reference's operation order).  Compiled without implicit
// multiply-add contraction: the kernels fuse where their source asks (fma,
// the paired FP32x2 intrinsics), so a kernel and its member-batched copy
// compute the same bits.
#include "orchestrate.cuh"

PLL_DEFINE_FORM(f32, float)
