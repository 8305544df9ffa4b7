// Stand-in for Source/PeleC.H in the oracle/_ref build: only what the hot-path headers
// take from it -- the AMReX shim, the index layout, and the PCPhysBCType numbering of
// Source/PeleC.H:49-57 (which matches amrex::PhysBCType with user_bc appended).
#pragma once
#include "pcg_amrex_shim.H"
#include "Constants.H"
#include "IndexDefines.H"

namespace PCPhysBCType {
enum phys_bc_type { interior = 0, inflow, outflow, symmetry, slip_wall, no_slip_wall, user_bc };
}
