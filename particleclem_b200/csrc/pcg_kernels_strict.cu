// FP64 parity kernels: compiled with --fmad=false so that every expression rounds as
// in the reference (and the CPU oracle), operation by operation. Built once per species
// count of the build (-DPCG_TU_NS=n, namespace pcg_strict<n>).
#define PCG_CAT2(a, b) a##b
#define PCG_CAT(a, b) PCG_CAT2(a, b)
#define PCG_TU PCG_CAT(pcg_strict, PCG_TU_NS)
#define PCG_TU_DOUBLE_ONLY
#include "pcg_dispatch.cuh"
