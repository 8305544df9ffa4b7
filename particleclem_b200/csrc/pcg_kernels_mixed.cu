// The mixed form's stage kernels (PCG_PREC_MIXED): FP32 trace, Riemann and transverse
// arithmetic, FP64 state, ctoprim Newton solve and flux accumulation. Built once per
// species count of the build (namespace pcg_mixed<n>), with FMA contraction and the approximate
// FP32 division and square root.
#define PCG_CAT2(a, b) a##b
#define PCG_CAT(a, b) PCG_CAT2(a, b)
#define PCG_TU PCG_CAT(pcg_mixed, PCG_TU_NS)
#define PCG_TU_SINGLE_ONLY
#include "pcg_dispatch.cuh"
