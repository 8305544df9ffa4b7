// Stand-in for Source/EB.H in the oracle/_ref build. Every cell is regular, so the only
// EB helper the Godunov sources reach, is_cut_neighborhood, is always false.
#pragma once
#include "pcg_amrex_shim.H"
#include "PeleC.H"
#include "IndexDefines.H"

inline bool
is_cut_neighborhood(
  const amrex::IntVect& /*iv*/,
  amrex::Array4<amrex::EBCellFlag const> const& /*flags*/,
  const amrex::IntVect& /*ng*/ = amrex::IntVect(1))
{
  return false;
}
