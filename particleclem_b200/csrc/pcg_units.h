// pcg_units.h -- the registry of kernel units. The species count of the reference is a
// compile-time constant of the mechanism (NUM_SPECIES, Source/IndexDefines.H:50-89), and
// so it is here: every kernel translation unit is compiled for ONE species count and one
// arithmetic, and registers its launch entry points at library load. The host routes a
// call to the unit of its (arithmetic, species count); the build decides which species
// counts exist (particleclem_b200/build.py, PCG_NSPEC).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "pcg_types.h"

namespace pcg {

enum UnitKind { UNIT_STRICT = 0, UNIT_FAST = 1, UNIT_MIXED = 2, UNIT_NKIND = 3 };

struct UnitEntry {
  int kind;  // UnitKind
  int ns;    // species count
  cudaError_t (*upload_eos)(int slot, const EosConst& e);
  cudaError_t (*launch_stage)(int stage, int ns, bool single, const StageArgs& a, int64_t nblocks, int variant,
                              cudaStream_t s);
  // FP64 step tail (strict and fast units), nullptr in the mixed units
  cudaError_t (*launch_advance)(int ns, const StageArgs& a, int64_t nblocks, int variant, cudaStream_t s);
  // FP64 auxiliary kernels (strict units only)
  cudaError_t (*launch_aux)(int which, int ns, const AuxArgs& a, int64_t nblocks, cudaStream_t s);
};

// Defined by the host unit; called from the static initialisers of the kernel units.
void register_unit(const UnitEntry& u);

}  // namespace pcg
