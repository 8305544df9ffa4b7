// pcg_dispatch.cuh -- per-translation-unit launch entry points. Included by
// pcg_kernels_strict.cu (FP64, --fmad=false) and pcg_kernels_fast.cu (FMA allowed),
// each with its own PCG_TU namespace and its own copy of the EOS constant bank.
#pragma once

#include <cuda_runtime.h>

#include "pcg_kernels.cuh"
#include "pcg_aux_kernels.cuh"

namespace PCG_TU {

// slot 0: gamma law, slot 1: NASA-7 mixture (synchronous upload).
cudaError_t upload_eos(int slot, const pcg::EosConst& e) {
  return cudaMemcpyToSymbol(c_eos, &e, sizeof(e), slot * sizeof(e), cudaMemcpyHostToDevice);
}

#ifdef PCG_TU_DOUBLE_ONLY
constexpr bool kExact = true;  // reference expression order
#else
constexpr bool kExact = false;  // reduced algebra
#endif

template <int NS, bool MIX, class R, int V>
static cudaError_t launch_v(int stage, const pcg::StageArgs& a, const dim3& grid, const dim3& block, cudaStream_t s) {
  switch (stage) {
    case K_CTOPRIM: k_ctoprim<NS, MIX, kMinBlocks[K_CTOPRIM][V]><<<grid, block, 0, s>>>(a); break;
    case K_PREP: k_prep<NS, MIX, kExact, R><<<grid, block, 0, s>>>(a); break;
    case K_TRACE:
      if (a.use_hybrid_weno && a.ppm_type == 1)
        k_trace_weno<NS, MIX, kExact, R><<<grid, block, 0, s>>>(a);  // one shape for every variant
      else
        k_trace<NS, MIX, kExact, R, kMinBlocks[K_TRACE][V]><<<grid, block, 0, s>>>(a);
      break;
    case K_FLUX0: k_flux0<NS, MIX, kExact, R, kMinBlocks[K_FLUX0][V]><<<grid, block, 0, s>>>(a); break;
    case K_FLUX1: k_flux1<NS, MIX, kExact, R, kMinBlocks[K_FLUX1][V]><<<grid, block, 0, s>>>(a); break;
    case K_FLUX2: k_flux2<NS, MIX, kExact, R, kMinBlocks[K_FLUX2][V]><<<grid, block, 0, s>>>(a); break;
    case K_CONSUP: k_consup<NS, MIX><<<grid, block, 0, s>>>(a); break;
    case K_LOWBC: k_lowbc<NS, MIX, kExact, R><<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int NS, bool MIX, class R>
static cudaError_t launch_t(int stage, const pcg::StageArgs& a, int64_t nblocks, int variant, cudaStream_t s) {
  if (nblocks <= 0) return cudaSuccess;
  const dim3 grid((unsigned)nblocks), block(128);
  switch (variant) {
    case 0: return launch_v<NS, MIX, R, 0>(stage, a, grid, block, s);
    case 1: return launch_v<NS, MIX, R, 1>(stage, a, grid, block, s);
    case 2: return launch_v<NS, MIX, R, 2>(stage, a, grid, block, s);
    default: return cudaErrorInvalidValue;
  }
}

// ns: species count (1: gamma law, 9: NASA-7 mixture); single: FP32 compute type.
cudaError_t launch_stage(int stage, int ns, bool single, const pcg::StageArgs& a, int64_t nblocks, int variant,
                         cudaStream_t s) {
#ifdef PCG_TU_DOUBLE_ONLY
  if (single) return cudaErrorInvalidValue;
  if (ns == 1) return launch_t<1, false, double>(stage, a, nblocks, variant, s);
  if (ns == 9) return launch_t<9, true, double>(stage, a, nblocks, variant, s);
#else
  if (ns == 1)
    return single ? launch_t<1, false, float>(stage, a, nblocks, variant, s)
                  : launch_t<1, false, double>(stage, a, nblocks, variant, s);
  if (ns == 9)
    return single ? launch_t<9, true, float>(stage, a, nblocks, variant, s)
                  : launch_t<9, true, double>(stage, a, nblocks, variant, s);
#endif
  return cudaErrorInvalidValue;
}

cudaError_t launch_advance(int ns, const pcg::StageArgs& a, int64_t nblocks, int variant, cudaStream_t s) {
  if (ns == 1) return launch_advance_t<1, false>(a, nblocks, variant, s);
  if (ns == 9) return launch_advance_t<9, true>(a, nblocks, variant, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_aux(int which, int ns, const pcg::AuxArgs& a, int64_t nblocks, cudaStream_t s) {
  if (ns == 1) return launch_aux_t<1, false>(which, a, nblocks, s);
  if (ns == 9) return launch_aux_t<9, true>(which, a, nblocks, s);
  return cudaErrorInvalidValue;
}

}  // namespace PCG_TU
