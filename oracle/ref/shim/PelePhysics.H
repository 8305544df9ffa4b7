// Stand-in for PelePhysics' EOS interface (pele::physics::PhysicsType::eos()) in the
// oracle/_ref build. Every method forwards to the oracle's documented EOS restatement
// (oracle/pcg_oracle.c), so the reference's own hydro sources and the oracle share one
// EOS definition and parity isolates the hydro algorithm.
#pragma once
#include "pcg_amrex_shim.H"
#include "mechanism.H"
#include "pcg_oracle.h"

namespace pele {
namespace physics {
namespace Constants {
constexpr amrex::Real RU = 8.31446261815324e7;
}
namespace eos {
struct SRK {};
struct Restated {
  void RPY2Cs(amrex::Real R, amrex::Real P, const amrex::Real* Y, amrex::Real& Cs) const { orc_eos_rpy2cs(R, P, Y, &Cs); }
  void RYP2E(amrex::Real R, const amrex::Real* Y, amrex::Real P, amrex::Real& E) const { orc_eos_ryp2e(R, Y, P, &E); }
  void REY2T(amrex::Real R, amrex::Real E, const amrex::Real* Y, amrex::Real& T) const { orc_eos_rey2t(R, E, Y, &T); }
  void RTY2P(amrex::Real R, amrex::Real T, const amrex::Real* Y, amrex::Real& P) const { orc_eos_rty2p(R, T, Y, &P); }
  void RTY2Cs(amrex::Real R, amrex::Real T, const amrex::Real* Y, amrex::Real& Cs) const { orc_eos_rty2cs(R, T, Y, &Cs); }
  void RTY2G(amrex::Real R, amrex::Real T, const amrex::Real* Y, amrex::Real& G) const { orc_eos_rty2g(R, T, Y, &G); }
  void RTY2dpde_dpdre(amrex::Real R, amrex::Real T, const amrex::Real* Y, amrex::Real& dpde, amrex::Real& dpdr_e) const {
    orc_eos_rty2dpde_dpdre(R, T, Y, &dpde, &dpdr_e);
  }
  void Y2WBAR(const amrex::Real* Y, amrex::Real& WBAR) const { orc_eos_y2wbar(Y, &WBAR); }
  void T2Ei(amrex::Real T, amrex::Real* Ei) const { orc_eos_t2ei(T, Ei); }
};
} // namespace eos
struct PhysicsType {
  using eos_type = eos::Restated;
  static eos_type eos() { return eos_type{}; }
};
} // namespace physics
} // namespace pele
