// FP64 kernels with FMA contraction (PCG_PREC_FP64_FAST), and the FP64 step tail both
// fast forms share. Built once per species count of the build (namespace pcg_fast<n>).
#define PCG_CAT2(a, b) a##b
#define PCG_CAT(a, b) PCG_CAT2(a, b)
#define PCG_TU PCG_CAT(pcg_fast, PCG_TU_NS)
#include "pcg_dispatch.cuh"
