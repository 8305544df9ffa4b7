// pcg_pelec_adapter.H -- the PeleC-side binding of libpcg_hydro.so (C++, header only).
//
// A PeleC build includes this header where Source/Hydro.cpp calls the Godunov path and
// replaces
//   pc_ctoprim's launch      (Source/Hydro.cpp:104-116) by pcg_ctoprim,
//   pc_srctoprim's launch    (Source/Hydro.cpp:161-174) by pcg_srctoprim,
//   pc_umdrv                 (Source/Hydro.cpp:245-249) by pcg_umdrv,
//   update_flux_registers    (Source/Hydro.cpp:281-287) and reflux
//                            (Source/PeleC.cpp:1403-1414) by the library's register,
// passing its FABs as pcg_array4 descriptors: same addressing as amrex::Array4, no
// copies. It needs only amrex::Array4, amrex::GpuArray and amrex::Real from AMReX (the
// repository's tests compile it against a small AMReX-API shim).
#ifndef PCG_PELEC_ADAPTER_H
#define PCG_PELEC_ADAPTER_H

#include "pcg_hydro.h"

namespace pcg_pelec {

// amrex::Array4 -> pcg_array4 (pointer, strides, index bounds, component count)
template <class T>
inline pcg_array4 to_array4(amrex::Array4<T> const& a) {
  pcg_array4 d;
  d.p = const_cast<double*>(static_cast<const double*>(a.dataPtr()));
  d.jstride = a.jstride;
  d.kstride = a.kstride;
  d.nstride = a.nstride;
  d.begin[0] = a.begin.x;
  d.begin[1] = a.begin.y;
  d.begin[2] = a.begin.z;
  d.end[0] = a.end.x;
  d.end[1] = a.end.y;
  d.end[2] = a.end.z;
  d.ncomp = a.ncomp;
  return d;
}

// The runtime parameters pc_umdrv receives (Source/Hydro.H:910-935).
inline pcg_hydro_params params(amrex::GpuArray<amrex::Real, 3> const& dx, amrex::Real dt, const int* domlo,
                               const int* domhi, const int* bclo, const int* bchi, int ppm_type, int plm_iorder,
                               bool use_flattening, bool use_hybrid_weno, int weno_scheme, amrex::Real difmag,
                               int nspec, int precision_mode = PCG_PREC_FP64) {
  pcg_hydro_params p{};
  for (int d = 0; d < 3; ++d) {
    p.dx[d] = dx[d];
    p.domlo[d] = domlo[d];
    p.domhi[d] = domhi[d];
    p.bclo[d] = bclo[d];
    p.bchi[d] = bchi[d];
  }
  p.dt = dt;
  p.difmag = difmag;
  p.ppm_type = ppm_type;
  p.plm_iorder = plm_iorder;
  p.use_flattening = use_flattening;
  p.use_hybrid_weno = use_hybrid_weno;
  p.weno_scheme = weno_scheme;
  p.nspec = nspec;
  p.precision_mode = precision_mode;
  return p;
}

// pc_umdrv's signature (Source/Hydro.H:910-935) on top of pcg_umdrv; time and cflLoc are
// unused by the reference as well. Returns PCG_OK or a PCG_E* code.
inline int umdrv(amrex::Box const& bx, const int* domlo, const int* domhi, const int* bclo, const int* bchi,
                 amrex::Array4<const amrex::Real> const& uin, amrex::Array4<amrex::Real> const& uout,
                 amrex::Array4<const amrex::Real> const& q, amrex::Array4<const amrex::Real> const& qaux,
                 amrex::Array4<const amrex::Real> const& src_q, amrex::GpuArray<amrex::Real, 3> const& dx,
                 amrex::Real dt, int ppm_type, int plm_iorder, bool use_flattening, bool use_hybrid_weno,
                 int weno_scheme, amrex::Real difmag, amrex::Array4<amrex::Real> const* flx,
                 amrex::Array4<const amrex::Real> const* a, amrex::Array4<amrex::Real> const& vol, int nspec,
                 pcg_stream_t stream) {
  const pcg_hydro_params prm = params(dx, dt, domlo, domhi, bclo, bchi, ppm_type, plm_iorder, use_flattening,
                                      use_hybrid_weno, weno_scheme, difmag, nspec);
  const int32_t lo[3] = {bx.smallEnd(0), bx.smallEnd(1), bx.smallEnd(2)};
  const int32_t hi[3] = {bx.bigEnd(0), bx.bigEnd(1), bx.bigEnd(2)};
  const pcg_array4 u = to_array4(uin), qq = to_array4(q), qa = to_array4(qaux), sq = to_array4(src_q),
                   vv = to_array4(vol);
  pcg_array4 uo = to_array4(uout);
  pcg_array4 fl[3], ar[3];
  for (int d = 0; d < 3; ++d) {
    fl[d] = to_array4(flx[d]);
    ar[d] = to_array4(a[d]);
  }
  return pcg_umdrv(&prm, lo, hi, &u, &uo, &qq, &qa, &sq, fl, ar, &vv, stream);
}

// PeleC::update_flux_registers (Source/PeleC.cpp:1343-1400) for regular boxes, on the
// library's register: fr_as_crse is the register of the level above (nullptr on the
// finest level), fr_as_fine the register of this level (nullptr on level 0). flux: the
// box's three area-weighted flux FABs. (The reference passes the cell volume as "dx";
// the library's calls take the area-weighted fluxes directly.)
inline int update_flux_registers(pcg_fluxreg* fr_as_crse, pcg_fluxreg* fr_as_fine, amrex::Box const& bx,
                                 amrex::Array4<const amrex::Real> const* flux, amrex::Real dt, pcg_stream_t stream) {
  const int32_t lo[3] = {bx.smallEnd(0), bx.smallEnd(1), bx.smallEnd(2)};
  const int32_t hi[3] = {bx.bigEnd(0), bx.bigEnd(1), bx.bigEnd(2)};
  const pcg_array4 f[3] = {to_array4(flux[0]), to_array4(flux[1]), to_array4(flux[2])};
  int rc = PCG_OK;
  if (fr_as_crse) rc = pcg_fluxreg_crse_add(fr_as_crse, lo, hi, f, dt, stream);
  if (rc == PCG_OK && fr_as_fine) rc = pcg_fluxreg_fine_add(fr_as_fine, lo, hi, f, dt, stream);
  return rc;
}

// PeleC::reflux (Source/PeleC.cpp:1403-1414) on one coarse FAB that holds every cell the
// register corrects; vol: the coarse cell volume.
inline int reflux(pcg_fluxreg* reg, amrex::Array4<amrex::Real> const& s_crse, amrex::Real vol, pcg_stream_t stream) {
  pcg_array4 s = to_array4(s_crse);
  return pcg_fluxreg_reflux(reg, &s, vol, stream);
}

}  // namespace pcg_pelec

#endif
