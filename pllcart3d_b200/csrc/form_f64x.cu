// The exact FP64 form of the step: the reference's arithmetic, operation by
// operation, compiled without multiply-add contraction (--fmad=false), the
// DCT sums in sequential order and every division the reference performs.
// Selected by exact_dct; the stages that call no exp() reproduce the CPU
// restatement bit for bit.
#define PLL_FP64_EXACT 1
#include "orchestrate.cuh"

PLL_DEFINE_FORM(f64x, double)
