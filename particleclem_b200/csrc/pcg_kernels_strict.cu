// FP64 parity kernels: compiled with --fmad=false so that every expression rounds as
// in the reference (and the CPU oracle), operation by operation.
#define PCG_TU pcg_strict
#define PCG_TU_DOUBLE_ONLY
#include "pcg_dispatch.cuh"
