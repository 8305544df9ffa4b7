// pcg_dispatch.cuh -- per-translation-unit launch entry points. Each kernel translation
// unit instantiates the stage kernels for ONE species count (PCG_TU_NS) and one
// arithmetic: PCG_TU_DOUBLE_ONLY (FP64 reference order, compiled --fmad=false),
// PCG_TU_SINGLE_ONLY (the mixed form's FP32 stage kernels) or neither (FP64 with FMA
// contraction, and the FP64 step tail of both fast forms). Each unit has its own
// PCG_TU namespace and its own copy of the EOS constant bank, and registers itself with
// the host (pcg_units.h), which routes a call to the unit of its (precision form,
// species count).
#pragma once

#include <cuda_runtime.h>

#include "pcg_kernels.cuh"
#include "pcg_aux_kernels.cuh"
#include "pcg_units.h"

#ifndef PCG_TU_NS
#error "PCG_TU_NS (species count of this translation unit) must be defined"
#endif

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

// pcg_umeth's final stage (raw fluxes and face states), its low-order boundary faces and
// p div u; pcg_srctoprim. One launch shape each.
template <int NS, bool MIX, class R>
static cudaError_t launch_special(int stage, const pcg::StageArgs& a, const dim3& grid, const dim3& block,
                                  cudaStream_t s) {
  switch (stage) {
    case K_FLUX2: k_flux2<NS, MIX, kExact, R, 0, true><<<grid, block, 0, s>>>(a); break;
    case K_LOWBC: k_lowbc<NS, MIX, kExact, R, true><<<grid, block, 0, s>>>(a); break;
    case K_CONSUP: k_pdivu<NS><<<grid, block, 0, s>>>(a); break;
    case K_SRCQ: k_srctoprim<NS><<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int NS, bool MIX, class R>
static cudaError_t launch_trace_tile(const pcg::StageArgs& a, const dim3& grid, const dim3& block, int variant,
                                    cudaStream_t s) {
  if constexpr (sizeof(R) == 4 && pcg::trace_tile_species(NS)) {
    switch (variant) {
      case 0: k_trace_tile<NS, MIX, kMinBlocks[K_TRACE][0]><<<grid, block, 0, s>>>(a); break;
      case 1: k_trace_tile<NS, MIX, kMinBlocks[K_TRACE][1]><<<grid, block, 0, s>>>(a); break;
      case 2: k_trace_tile<NS, MIX, kMinBlocks[K_TRACE][2]><<<grid, block, 0, s>>>(a); break;
      default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
  } else {
    return cudaErrorInvalidValue;  // the FP64 forms and large species counts trace per cell
  }
}

template <int NS, bool MIX, class R>
static cudaError_t launch_t(int stage, const pcg::StageArgs& a, int64_t nblocks, int variant, cudaStream_t s) {
  if (nblocks <= 0) return cudaSuccess;
  const dim3 grid((unsigned)nblocks), block(128);
  if (stage == K_TRACE_TILE) return launch_trace_tile<NS, MIX, R>(a, grid, block, variant, s);
  if (stage == K_SRCQ || (a.umeth && (stage == K_FLUX2 || stage == K_LOWBC || stage == K_CONSUP)))
    return launch_special<NS, MIX, R>(stage, a, grid, block, s);
  switch (variant) {
    case 0: return launch_v<NS, MIX, R, 0>(stage, a, grid, block, s);
    case 1: return launch_v<NS, MIX, R, 1>(stage, a, grid, block, s);
    case 2: return launch_v<NS, MIX, R, 2>(stage, a, grid, block, s);
    default: return cudaErrorInvalidValue;
  }
}

// ns: species count (1: gamma law, more: NASA-7 mixture); single: FP32 compute type. A
// combination this unit does not hold is cudaErrorInvalidValue.
constexpr int kNS = PCG_TU_NS;
constexpr bool kMix = PCG_TU_NS > 1;

cudaError_t launch_stage(int stage, int ns, bool single, const pcg::StageArgs& a, int64_t nblocks, int variant,
                         cudaStream_t s) {
  if (ns != kNS) return cudaErrorInvalidValue;
#if defined(PCG_TU_DOUBLE_ONLY)
  if (single) return cudaErrorInvalidValue;
  return launch_t<kNS, kMix, double>(stage, a, nblocks, variant, s);
#elif defined(PCG_TU_SINGLE_ONLY)
  if (!single) return cudaErrorInvalidValue;
  return launch_t<kNS, kMix, float>(stage, a, nblocks, variant, s);
#else
  if (single) return cudaErrorInvalidValue;
  return launch_t<kNS, kMix, double>(stage, a, nblocks, variant, s);
#endif
}

#if !defined(PCG_TU_SINGLE_ONLY)
cudaError_t launch_advance(int ns, const pcg::StageArgs& a, int64_t nblocks, int variant, cudaStream_t s) {
  if (ns != kNS) return cudaErrorInvalidValue;
  return launch_advance_t<kNS, kMix>(a, nblocks, variant, s);
}
#endif

#if defined(PCG_TU_DOUBLE_ONLY)
cudaError_t launch_aux(int which, int ns, const pcg::AuxArgs& a, int64_t nblocks, cudaStream_t s) {
  if (ns != kNS) return cudaErrorInvalidValue;
  return launch_aux_t<kNS, kMix>(which, a, nblocks, s);
}
#endif

// Registration with the host's unit table at library load.
struct UnitRegistration {
  UnitRegistration() {
    pcg::UnitEntry u{};
    u.ns = kNS;
    u.upload_eos = &upload_eos;
    u.launch_stage = &launch_stage;
#if defined(PCG_TU_DOUBLE_ONLY)
    u.kind = pcg::UNIT_STRICT;
    u.launch_advance = &launch_advance;
    u.launch_aux = &launch_aux;
#elif defined(PCG_TU_SINGLE_ONLY)
    u.kind = pcg::UNIT_MIXED;
#else
    u.kind = pcg::UNIT_FAST;
    u.launch_advance = &launch_advance;
#endif
    pcg::register_unit(u);
  }
};
static UnitRegistration g_unit_registration;

}  // namespace PCG_TU
