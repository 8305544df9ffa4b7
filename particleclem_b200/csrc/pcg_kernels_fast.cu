// Fast kernels: FP64 with FMA contraction, and the mixed form (FP32 trace/Riemann/
// transverse arithmetic, FP64 state, update, Newton and dt).
#define PCG_TU pcg_fast
#include "pcg_dispatch.cuh"
