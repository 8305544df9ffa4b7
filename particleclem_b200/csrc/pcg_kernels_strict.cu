// FP64 parity kernels: compiled with --fmad=false so that every expression rounds as
// in the reference (and the CPU oracle), operation by operation. Built once per species
// count (-DPCG_TU_NS=1 / 9) into namespaces pcg_strict1 / pcg_strict9.
#define PCG_CAT2(a, b) a##b
#define PCG_CAT(a, b) PCG_CAT2(a, b)
#define PCG_TU PCG_CAT(pcg_strict, PCG_TU_NS)
#define PCG_TU_DOUBLE_ONLY
#include "pcg_dispatch.cuh"
