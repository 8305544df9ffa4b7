// pcg_kernels.cuh -- the stage kernels of the batched Godunov advance.
//
// One launch per stage covers every box of a batch: the launch's blocks are split
// into segments (one region and one variant each, see pcg::Seg) so that uneven boxes
// share a launch. Stages:
//   K_CTOPRIM  pc_ctoprim on grow(box,4)                              -> q, qaux
//   K_PREP     per cell of grow(box,1): shock flattening (3 directions) and the
//              cell sound speed the trace uses; per node of the box: div u      -> prep, divu
//   K_TRACE    trace_ppm / PLM, one direction per thread, grow(box,1)   -> trm[d], trp[d]
//   K_FLUX0    first Riemann solve in each direction                    -> fi[d]
//   K_FLUX1    pc_transdo + Riemann for both transverse partners of d  -> fdo[d][o]
//   K_FLUX2    pc_transdd + final Riemann + pc_artif_visc + pc_norm_spec_flx
//              + pc_ext_flx                                             -> ff[d], qec[d]
//   K_LOWBC    pc_low_order_boundary: inflow/user_bc domain faces again from
//              PLM states without transverse terms, after K_FLUX2      -> ff[d], qec[d]
//   K_CONSUP   pc_pdivu + pc_update                                     -> uout
// Traced states are kept only for the cells whose states reach the box's fluxes
// (grow(box,1)); the reference traces grow(box,2), whose outer layer feeds no output.
// The per-cell quantities the reference recomputes in each of its three trace passes
// (flatten, the cell sound speed) are computed once. EXACT selects the reference
// expression order (parity form) or the reduced algebra (FMA / mixed forms).
#pragma once

#include "pcg_device.cuh"
#include "pcg_tma.cuh"

namespace PCG_TU {

enum { K_CTOPRIM = 0, K_PREP, K_TRACE, K_FLUX0, K_FLUX1, K_FLUX2, K_CONSUP, K_NSTAGE };
// launches that are not stages of their own: the inflow/user_bc boundary faces (within
// stage K_FLUX2), pc_srctoprim (pcg_srctoprim) and the TMA-staged trace (stage K_TRACE of
// the mixed form)
enum { K_LOWBC = K_NSTAGE, K_SRCQ, K_TRACE_TILE };

// Launch variants: each heavy stage is compiled with a few minimum-resident-blocks
// requests (__launch_bounds__ register caps); the host picks one per (form, species
// count, stage) from a table the autotuner fills. 0 = no cap.
constexpr int kMinBlocks[K_NSTAGE][3] = {
  {0, 5, 8},  // ctoprim
  {0, 0, 0},  // prep
  {0, 4, 5},  // trace
  {0, 6, 8},  // flux0
  {5, 6, 8},  // flux1
  {4, 5, 6},  // flux2
  {0, 5, 6},  // consup: the caps apply to the fused step tail (k_advance)
};

struct Item {
  const pcg::Region* rg;
  int variant;
  int i, j, k;
};

// Timestep of a region and the constants the reference derives from it
// (Source/Godunov.cpp:85-91, Source/PPM.cpp:37), with the same expressions.
__device__ __forceinline__ double dt_of(const pcg::StageArgs& a, const pcg::Region& rg) {
  return a.dt_dev ? *a.dt_dev : rg.dt_ptr ? *rg.dt_ptr : rg.dt;
}

// Segment counts and block numbers stay below 2^31 (the host checks the launch sizes),
// so the thread's position is formed with 32-bit (unsigned) division.
__device__ __forceinline__ bool item_of(const pcg::StageArgs& a, Item& it) {
  const int blk = blockIdx.x;
  int lo = 0, hi = a.nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.segs[mid].blk0 <= blk) lo = mid; else hi = mid - 1;
  }
  const pcg::Seg& s = a.segs[lo];
  const unsigned local = unsigned(blk - (int)s.blk0) * blockDim.x + threadIdx.x;
  if (local >= (unsigned)s.count) return false;
  const unsigned n0 = s.n[0], n1 = s.n[1];
  const unsigned t = local / n0;
  it.i = s.lo[0] + (int)(local - t * n0);
  it.j = s.lo[1] + (int)(t % n1);
  it.k = s.lo[2] + (int)(t / n1);
  it.rg = a.regions + s.region;
  it.variant = s.variant;
  return true;
}

// The segment of this block and the block's index within it (tiled stages).
__device__ __forceinline__ const pcg::Seg& seg_of(const pcg::StageArgs& a, int& local_block) {
  const int blk = blockIdx.x;
  int lo = 0, hi = a.nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.segs[mid].blk0 <= blk) lo = mid; else hi = mid - 1;
  }
  local_block = blk - (int)a.segs[lo].blk0;
  return a.segs[lo];
}

// A pointer positioned at one cell of a view: components n at p[n * ns].
template <class T>
struct CellPtr {
  T* p;
  int ns;
  __device__ __forceinline__ T& operator[](int n) const { return p[n * ns]; }
};
template <class T>
__device__ __forceinline__ CellPtr<T> at(const V4<T>& v, int i, int j, int k) {
  return CellPtr<T>{&v(i, j, k, 0), v.ns};
}
template <class T>
__device__ __forceinline__ CellPtr<T> shift(const CellPtr<T>& c, int off) {
  return CellPtr<T>{c.p + off, c.ns};
}
template <class T>
__device__ __forceinline__ int dstride(const V4<T>& v, int d) {
  return d == 0 ? 1 : d == 1 ? v.js : v.ks;
}
// One cell of a blocked view: component n at p[n * kCellBlock] (a compile-time offset).
template <class T>
struct BCell {
  T* p;
  __device__ __forceinline__ T& operator[](int n) const { return p[n * pcg::kCellBlock]; }
};
template <class T>
__device__ __forceinline__ BCell<T> at(const B4<T>& v, int i, int j, int k) {
  return BCell<T>{v.cell(i, j, k)};
}
// the neighbour of (i, j, k) one cell up in direction d
template <class T>
__device__ __forceinline__ BCell<T> at_up(const B4<T>& v, int i, int j, int k, int d) {
  return at(v, i + (d == 0), j + (d == 1), k + (d == 2));
}

// The pressure offset of a region for the FP32 arithmetic (see PDev): the ideal-gas
// pressure RU * sum(rhoY_k / W_k) * T of the region's first valid cell, from the
// conserved partial densities and the stored temperature (any constant of the region
// would do; this one needs no neighbour, no division and no Newton solve, so every
// stage computes the same value cheaply); zero for FP64.
// A region without a conserved state (pcg_umeth, which takes only q and qaux) uses the
// primitive pressure of the same cell.
template <int NS, bool MIX, class R>
__device__ __forceinline__ double p0_of(const pcg::Region& rg) {
  if constexpr (PDev<R>::on) {
    if (!rg.uin.p) return v4<const double>(rg.q)(rg.lo[0], rg.lo[1], rg.lo[2], pcg::QPRES);
    const CellPtr<const double> u{&v4<const double>(rg.uin)(rg.lo[0], rg.lo[1], rg.lo[2], 0), rg.uin.ns};
    double w[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) w[n] = u[pcg::UFS + n];
    return Eos<NS, MIX, double>::rmix(w) * u[pcg::UTEMP];
  } else {
    return 0.0;
  }
}

// ------------------------------------------------------------------ ctoprim
// Source/PeleCUtilities.H:242-320 (pc_ctoprim), omega = rad = 0.
template <int NS, bool MIX, int MINB>
__global__ void __launch_bounds__(128, MINB) k_ctoprim(pcg::StageArgs a) {
  Item it;
  if (!item_of(a, it)) return;
  const pcg::Region& rg = *it.rg;
  using E = Eos<NS, MIX, double>;
  const CellPtr<const double> u = at(v4<const double>(rg.uin), it.i, it.j, it.k);
  const CellPtr<double> qa = at(v4<double>(rg.qa), it.i, it.j, it.k);
  const double rho = u[pcg::URHO];
  const double rhoinv = 1.0 / rho;
  const double vx = u[pcg::UMX] * rhoinv;
  const double vy = u[pcg::UMY] * rhoinv;
  const double vz = u[pcg::UMZ] * rhoinv;
  const double kineng = 0.5 * rho * (vx * vx + vy * vy + vz * vz) - 0.5 * rho * 0.0 * 0.0 * 0.0 * 0.0;
  double y[NS];
#pragma unroll
  for (int n = 0; n < NS; n++) {
    double yn = u[pcg::UFS + n] / rho;
    if ((-1e-4 * DBL_EPSILON < yn) && (yn < 1e-4 * DBL_EPSILON)) yn = 0.0;
    y[n] = yn;
  }
  const double e = (u[pcg::UEDEN] - kineng) * rhoinv;
  const double wbar = E::y2wbar(y);
  const double T = E::rey2t(e, y, u[pcg::UTEMP]);
  double p, cs, gam1, dpde, dpdr_e;
  E::rty2all(rho, T, y, p, cs, gam1, dpde, dpdr_e);
  // the FP64 primitive array exists in the FP64 forms; the mixed form's stages read the
  // FP32 copy below instead
  if (rg.q.p) {
    const CellPtr<double> q = at(v4<double>(rg.q), it.i, it.j, it.k);
    q[pcg::QRHO] = rho;
    q[pcg::QU] = vx;
    q[pcg::QV] = vy;
    q[pcg::QW] = vz;
#pragma unroll
    for (int n = 0; n < NS; n++) q[pcg::QFS + n] = y[n];
    q[pcg::QTEMP] = T;
    q[pcg::QREINT] = e * rho;
    q[pcg::QPRES] = p;
    q[pcg::QGAME] = p / (e * rho) + 1.0;
  }
  qa[pcg::QDPDR] = dpdr_e;
  qa[pcg::QDPDE] = dpde;
  qa[pcg::QGAMC] = gam1;
  qa[pcg::QC] = cs;
  qa[pcg::QCSML] = dmax(pcg::SMALL_NUM, pcg::SMALL_NUM * cs);
  qa[pcg::QRSPEC] = pcg::RU / wbar;
  // mixed form: the FP32 primitive copy the trace reads, on grow(box, qf_grow)
  const int gq = rg.qf_grow;
  if (rg.qf.p && !rg.qf_in_prep && it.i >= rg.lo[0] - gq && it.i <= rg.hi[0] + gq && it.j >= rg.lo[1] - gq &&
      it.j <= rg.hi[1] + gq && it.k >= rg.lo[2] - gq && it.k <= rg.hi[2] + gq) {
    const double p0 = p0_of<NS, MIX, float>(rg);
    const CellPtr<float> f = at(v4<float>(rg.qf), it.i, it.j, it.k);
    f[pcg::TR_RHO] = float(rho);
    f[pcg::TR_U] = float(vx);
    f[pcg::TR_V] = float(vy);
    f[pcg::TR_W] = float(vz);
    f[pcg::TR_P] = float(p - p0);
    f[pcg::TR_RE] = float(e * rho);
#pragma unroll
    for (int n = 0; n < NS; ++n) f[pcg::TR_Y + n] = float(y[n]);
  }
}

// ------------------------------------------------------------------ prep
// The component of the trace-state layout (FP32 primitive copy) holding QVAR component
// qcomp.
__device__ __forceinline__ int tr_comp(int qcomp) {
  return qcomp == pcg::QRHO ? pcg::TR_RHO
         : qcomp <= pcg::QW ? pcg::TR_U + (qcomp - pcg::QU)
         : qcomp == pcg::QPRES ? pcg::TR_P
         : qcomp == pcg::QREINT ? pcg::TR_RE
                                : pcg::TR_Y + (qcomp - pcg::QFS);
}

// Primitive component qcomp of cell (i,j,k) read from the FP32 copy qf (trace-state
// layout), the pressure back to absolute (deviation + p0), as type T: what prep reads in
// the mixed form, where ctoprim writes no FP64 primitive array.
template <class T>
struct QfPrim {
  V4<const float> f;
  float p0;
  __device__ __forceinline__ T operator()(int i, int j, int k, int qcomp) const {
    const float v = f(i, j, k, tr_comp(qcomp));
    return qcomp == pcg::QPRES ? T(v) + T(p0) : T(v);
  }
};

// Source/Hydro.H:476-517 (pc_divu) at node (i,j,k); q any accessor of the primitives
template <class Q>
__device__ __forceinline__ double divu_node(const Q& q, int i, int j, int k, const double* dx) {
  const double ux = 0.25 *
                    (q(i, j, k, pcg::QU) - q(i - 1, j, k, pcg::QU) + q(i, j, k - 1, pcg::QU) -
                     q(i - 1, j, k - 1, pcg::QU) + q(i, j - 1, k, pcg::QU) - q(i - 1, j - 1, k, pcg::QU) +
                     q(i, j - 1, k - 1, pcg::QU) - q(i - 1, j - 1, k - 1, pcg::QU)) /
                    dx[0];
  const double vy = 0.25 *
                    (q(i, j, k, pcg::QV) - q(i, j - 1, k, pcg::QV) + q(i, j, k - 1, pcg::QV) -
                     q(i, j - 1, k - 1, pcg::QV) + q(i - 1, j, k, pcg::QV) - q(i - 1, j - 1, k, pcg::QV) +
                     q(i - 1, j, k - 1, pcg::QV) - q(i - 1, j - 1, k - 1, pcg::QV)) /
                    dx[1];
  const double wz = 0.25 *
                    (q(i, j, k, pcg::QW) - q(i, j, k - 1, pcg::QW) + q(i - 1, j, k, pcg::QW) -
                     q(i - 1, j, k - 1, pcg::QW) + q(i, j - 1, k, pcg::QW) - q(i, j - 1, k - 1, pcg::QW) +
                     q(i - 1, j - 1, k, pcg::QW) - q(i - 1, j - 1, k - 1, pcg::QW)) /
                    dx[2];
  return ux + vy + wz;
}

// Flattening, the trace's sound speed and the nodal div u of one cell of grow(box,1):
// q is the accessor the flattening and the sound speed read, qd the one div u reads.
template <int NS, bool MIX, bool EXACT, class R, class Q, class QD>
__device__ __forceinline__ void prep_cell(const pcg::StageArgs& a, const pcg::Region& rg, int i, int j, int k,
                                          const Q& q, const QD& qd) {
  R flat = R(1);
  if (a.use_flattening) {
#pragma unroll
    for (int df = 0; df < 3; df++) flat = dmin(flat, flatten<R>(q, i, j, k, df));
  }
  R cc;
  if (a.ppm_type == 1) {
    R y[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) y[n] = R(q(i, j, k, pcg::QFS + n));
    const R rho = R(q(i, j, k, pcg::QRHO)), p = R(q(i, j, k, pcg::QPRES));
    cc = EXACT ? Eos<NS, MIX, R>::rpy2cs(rho, p, y) : EosR<NS, MIX, R>::cs_y(rho, p, y);
  } else {
    cc = R(v4<const double>(rg.qa)(i, j, k, pcg::QC));
  }
  const CellPtr<R> pr = at(v4<R>(rg.prep), i, j, k);
  pr[0] = flat;
  pr[1] = cc;
  if (i >= rg.lo[0] && i <= rg.hi[0] + 1 && j >= rg.lo[1] && j <= rg.hi[1] + 1 && k >= rg.lo[2] && k <= rg.hi[2] + 1)
    v4<double>(rg.divu)(i, j, k) = divu_node(qd, i, j, k, rg.dx);
}

// prep components: 0 = flattening (min over the 3 directions, Source/PPM.cpp:108-115),
// 1 = sound speed the trace uses (PPM: RPY2Cs, Source/PPM.cpp:101; PLM: qaux QC). The
// flattening is evaluated in the compute type R: FP64 in the FP64 forms, FP32 in the
// mixed form (the primitive values rounded to FP32; it departs from 1 only at shocks).
template <int NS, bool MIX, bool EXACT, class R>
__global__ void __launch_bounds__(128) k_prep(pcg::StageArgs a) {
  Item it;
  if (!item_of(a, it)) return;
  const pcg::Region& rg = *it.rg;
  const int i = it.i, j = it.j, k = it.k;
  const V4<const double> q = v4<const double>(rg.q);
  if constexpr (PDev<R>::on) if (rg.qf_in_prep) {
    // FP32 copy of the primitive state for the trace (grow(box,3)), when the caller
    // supplied q (pcg_umdrv) and no ctoprim stage runs
    const double p0 = p0_of<NS, MIX, R>(rg);
    const CellPtr<const double> qc = at(q, i, j, k);
    const CellPtr<float> f = at(v4<float>(rg.qf), i, j, k);
    f[pcg::TR_RHO] = float(qc[pcg::QRHO]);
    f[pcg::TR_U] = float(qc[pcg::QU]);
    f[pcg::TR_V] = float(qc[pcg::QV]);
    f[pcg::TR_W] = float(qc[pcg::QW]);
    f[pcg::TR_P] = float(qc[pcg::QPRES] - p0);
    f[pcg::TR_RE] = float(qc[pcg::QREINT]);
#pragma unroll
    for (int n = 0; n < NS; ++n) f[pcg::TR_Y + n] = float(qc[pcg::QFS + n]);
  }
  const bool in_g1 = i >= rg.lo[0] - 1 && i <= rg.hi[0] + 1 && j >= rg.lo[1] - 1 && j <= rg.hi[1] + 1 &&
                     k >= rg.lo[2] - 1 && k <= rg.hi[2] + 1;
  if (!in_g1) return;
  if constexpr (PDev<R>::on) {
    if (!rg.q.p) {  // mixed form after ctoprim: only the FP32 copy exists
      const V4<const float> f = v4<const float>(rg.qf);
      const float p0 = float(p0_of<NS, MIX, R>(rg));
      prep_cell<NS, MIX, EXACT, R>(a, rg, i, j, k, QfPrim<R>{f, p0}, QfPrim<double>{f, p0});
      return;
    }
  }
  prep_cell<NS, MIX, EXACT, R>(a, rg, i, j, k, q, q);
}

// ------------------------------------------------------------------ trace
// The primitive state the trace reads: q itself (double, QVAR layout) in the FP64
// forms; in the mixed form the FP32 copy qf written by k_prep (trace-state layout,
// pressure as the deviation from the box's p0), so no conversions are left in the trace.
template <class R> struct Prim;
template <> struct Prim<double> {
  static constexpr bool kEdges = false;  // no precomputed PPM interface values
  const double* p;
  int ns, st;
  __device__ __forceinline__ Prim(const pcg::Region& rg, int i, int j, int k, int d) {
    const V4<const double> v = v4<const double>(rg.q);
    p = &v(i, j, k, 0);
    ns = v.ns;
    st = dstride(v, d);
  }
  __device__ __forceinline__ double c(int qcomp) const { return p[qcomp * ns]; }
  __device__ __forceinline__ void five(int qcomp, double* s) const { stencil<2>(qcomp, s); }
  template <int W>
  __device__ __forceinline__ void stencil(int qcomp, double* s) const {
    const double* b = p + qcomp * ns;
#pragma unroll
    for (int o = -W; o <= W; ++o) s[o + W] = b[o * st];
  }
};
template <> struct Prim<float> {
  static constexpr bool kEdges = false;
  const float* p;
  int ns, st;
  __device__ __forceinline__ Prim(const pcg::Region& rg, int i, int j, int k, int d) {
    const V4<const float> v = v4<const float>(rg.qf);
    p = &v(i, j, k, 0);
    ns = v.ns;
    st = dstride(v, d);
  }
  __device__ __forceinline__ float c(int qcomp) const { return p[tr_comp(qcomp) * ns]; }
  __device__ __forceinline__ void five(int qcomp, float* s) const { stencil<2>(qcomp, s); }
  template <int W>
  __device__ __forceinline__ void stencil(int qcomp, float* s) const {
    const float* b = p + tr_comp(qcomp) * ns;
#pragma unroll
    for (int o = -W; o <= W; ++o) s[o + W] = b[o * st];
  }
};

// Edge values sm, sp and centre value sc of component qcomp of the cell for the PPM
// trace: the PPM parabola (Source/PPM.H:28-115), or with HYB the hybrid-WENO edge values
// of Source/PPM.cpp:120-172 (weno_scheme 0 WENO-JS5, 1 WENO-Z5, 2 WENO-Z7, 3 WENO-Z3,
// any other value the PPM parabola).
template <bool HYB, class R, class PT>
__device__ __forceinline__ void ppm_edges(const PT& P, int qcomp, R flat, int scheme, R& sm, R& sp, R& sc) {
  if constexpr (PT::kEdges && !HYB) {
    // the accessor holds the interface values of the parabola (ppm_edge), formed once
    // per interface: only flattening and the limiter remain per cell
    P.edges(qcomp, sm, sp);
    sc = P.c(qcomp);
    ppm_limit<R>(sc, flat, sm, sp);
    return;
  }
  if constexpr (HYB) {
    if (scheme == 2) {
      R s7[7];
      P.template stencil<3>(qcomp, s7);
      weno::weno7z<R>(s7, sm, sp);
      sc = s7[3];
      return;
    }
    if (scheme == 3) {
      R s3[3];
      P.template stencil<1>(qcomp, s3);
      weno::weno3z<R>(s3, sm, sp);
      sc = s3[1];
      return;
    }
  }
  R s[5];
  P.five(qcomp, s);
  if (HYB && (scheme == 0 || scheme == 1))
    weno::weno5<R>(s, scheme == 1, sm, sp);
  else
    ppm_reconstruct<R>(s[0], s[1], s[2], s[3], s[4], flat, sm, sp);
  sc = s[2];
}

// Source/PPM.cpp:82-423 for one cell and direction D (bx == vbx as called from
// Source/Godunov.cpp:188-200, so both states are produced). Only the components the
// path reads are reconstructed: QGAME, QREINT and QTEMP profiles feed nothing.
// P: the primitive state around the cell (Prim: the global array; PrimTile: a staged
// shared-memory tile), with c(q), five(q, s) and stencil<W>(q, s) along D.
template <int NS, bool MIX, bool EXACT, bool HYB, int D, class R, class PT>
__device__ __forceinline__ void trace_ppm_dir(const pcg::Region& rg, const PT& P, int i, int j, int k, R cc, R flat,
                                              double dt, int scheme) {
  using E = Eos<NS, MIX, R>;
  using ER = EosR<NS, MIX, R>;
  const R dtdx = R(dt / rg.dx[D]);
  const R un = P.c(pcg::QU + D);
  R sm, sp, sc, s6;
  R Imr[3], Ipr[3], Imu[3], Ipu[3], Imp[3], Ipp[3];
  R Imt[3], Ipt[3];
  const R sp3[3] = {un - cc, un, un + cc};
  const R p0 = R(p0_of<NS, MIX, R>(rg));
#define PROFILE3(comp, Im, Ip)                                      \
  ppm_edges<HYB, R>(P, comp, flat, scheme, sm, sp, sc);              \
  s6 = ppm_s6<R>(sm, sp, sc);                                        \
  _Pragma("unroll") for (int w = 0; w < 3; ++w) ppm_wave<R>(sm, sp, s6, sp3[w], dtdx, Ip[w], Im[w]);
  PROFILE3(pcg::QRHO, Imr, Ipr)
  PROFILE3(pcg::QU + D, Imu, Ipu)
  PROFILE3(pcg::QPRES, Imp, Ipp)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (c == D) continue;
    ppm_edges<HYB, R>(P, pcg::QU + c, flat, scheme, sm, sp, sc);
    s6 = ppm_s6<R>(sm, sp, sc);
    ppm_wave<R>(sm, sp, s6, un, dtdx, Ipt[c], Imt[c]);
  }
  R ym0[NS], ym1[NS], yp1[NS], yp2[NS];
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    R Im[3], Ip[3];
    PROFILE3(pcg::QFS + n, Im, Ip)
    ym0[n] = Im[0];
    ym1[n] = Im[1];
    yp1[n] = Ip[1];
    yp2[n] = Ip[2];
  }
#undef PROFILE3
  const BCell<R> qp = at(b4<R>(rg.trp[D]), i, j, k);
  const BCell<R> qm = at(b4<R>(rg.trm[D]), i + (D == 0), j + (D == 1), k + (D == 2));
  // plus state on face i (Source/PPM.cpp:232-331)
  {
    R rho_ref = Imr[0];
    const R un_ref = Imu[0];
    R p_ref = Imp[0];
    rho_ref = dmax(rho_ref, Lim<R>::tiny());
    const R rho_ref_inv = R(1) / rho_ref;
    p_ref = dmax(p_ref, pfloor(Lim<R>::tiny(), p0));
    const R cc_ref = EXACT ? E::rpy2cs(rho_ref, p_ref, ym0) : ER::cs_y(rho_ref, pabs(p_ref, p0), ym0);
    const R csq_ref = cc_ref * cc_ref;
    const R cc_ref_inv = R(1) / cc_ref;
    const R dum = un_ref - Imu[0];
    const R dptotm = p_ref - Imp[0];
    const R drho = rho_ref - Imr[1];
    const R dptot = p_ref - Imp[1];
    const R dup = un_ref - Imu[2];
    const R dptotp = p_ref - Imp[2];
    R alpham = R(0.5) * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
    R alphap = R(0.5) * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
    R alpha0r = drho - (EXACT ? dptot / csq_ref : dptot * cc_ref_inv * cc_ref_inv);
    alpham = un - cc > R(0) ? R(0) : -alpham;
    alphap = un + cc > R(0) ? R(0) : -alphap;
    alpha0r = un > R(0) ? R(0) : -alpha0r;
    const R rhos = dmax(Lim<R>::tiny(), rho_ref + alphap + alpham + alpha0r);
    const R uns = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
    const R ps = dmax(pfloor(Lim<R>::tiny(), p0), p_ref + (alphap + alpham) * csq_ref);
    qp[pcg::TR_RHO] = rhos;
#pragma unroll
    for (int c = 0; c < 3; ++c) qp[pcg::TR_U + c] = (c == D) ? uns : Imt[c];
    qp[pcg::TR_P] = ps;
#pragma unroll
    for (int n = 0; n < NS; ++n) qp[pcg::TR_Y + n] = ym1[n];
    qp[pcg::TR_RE] = EXACT ? rhos * E::ryp2e(rhos, ym1, ps) : ER::rhoe_y(rhos, pabs(ps, p0), ym1);
  }
  // minus state on face i+1 (Source/PPM.cpp:334-422)
  {
    R rho_ref = Ipr[2];
    const R un_ref = Ipu[2];
    R p_ref = Ipp[2];
    rho_ref = dmax(rho_ref, Lim<R>::tiny());
    const R rho_ref_inv = R(1) / rho_ref;
    p_ref = dmax(p_ref, pfloor(Lim<R>::tiny(), p0));
    const R cc_ref = EXACT ? E::rpy2cs(rho_ref, p_ref, yp2) : ER::cs_y(rho_ref, pabs(p_ref, p0), yp2);
    const R csq_ref = cc_ref * cc_ref;
    const R cc_ref_inv = R(1) / cc_ref;
    const R dum = un_ref - Ipu[0];
    const R dptotm = p_ref - Ipp[0];
    const R drho = rho_ref - Ipr[1];
    const R dptot = p_ref - Ipp[1];
    const R dup = un_ref - Ipu[2];
    const R dptotp = p_ref - Ipp[2];
    R alpham = R(0.5) * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
    R alphap = R(0.5) * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
    R alpha0r = drho - (EXACT ? dptot / csq_ref : dptot * cc_ref_inv * cc_ref_inv);
    alpham = un - cc > R(0) ? -alpham : R(0);
    alphap = un + cc > R(0) ? -alphap : R(0);
    alpha0r = un > R(0) ? -alpha0r : R(0);
    const R rhos = dmax(Lim<R>::tiny(), rho_ref + alphap + alpham + alpha0r);
    const R uns = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
    const R ps = dmax(pfloor(Lim<R>::tiny(), p0), p_ref + (alphap + alpham) * csq_ref);
    qm[pcg::TR_RHO] = rhos;
#pragma unroll
    for (int c = 0; c < 3; ++c) qm[pcg::TR_U + c] = (c == D) ? uns : Ipt[c];
    qm[pcg::TR_P] = ps;
#pragma unroll
    for (int n = 0; n < NS; ++n) qm[pcg::TR_Y + n] = yp1[n];
    qm[pcg::TR_RE] = EXACT ? rhos * E::ryp2e(rhos, yp1, ps) : ER::rhoe_y(rhos, pabs(ps, p0), yp1);
  }
}

// A traced state held in registers (the low-order boundary faces).
template <class R>
struct RegState {
  R* a;
  __device__ __forceinline__ R& operator[](int n) const { return a[n]; }
};

// Source/PLM.H:167-309 (pc_plm_d) with the slopes of Source/Godunov.cpp:139-180, for the
// cell (i, j, k) and direction D: qp receives the state on the cell's low D-face (the
// right state of that face), qm the state on its high D-face (the left state there).
template <int NS, bool MIX, int D, class R, class QP, class QM, class PT>
__device__ __forceinline__ void plm_cell_p(const pcg::Region& rg, const PT& P, R cc, R flat, int order, double dt,
                                           const QP& qp, const QM& qm) {
  constexpr int l1 = (D == 0) ? 1 : 0;
  constexpr int l2 = (D == 2) ? 1 : 2;
  R s[5];
  const R p0 = R(p0_of<NS, MIX, R>(rg));
#define SLOPE(comp) (P.five(comp, s), plm_slope<R>(s[0], s[1], s[2], s[3], s[4], flat, order))
  const R drho = SLOPE(pcg::QRHO);
  const R dvel[3] = {SLOPE(pcg::QU), SLOPE(pcg::QV), SLOPE(pcg::QW)};
  const R dp = SLOPE(pcg::QPRES);
  const R drhoe = SLOPE(pcg::QREINT);
  const R dtdx = R(dt / rg.dx[D]);
  const R cs = cc * cc;
  const R rho = P.c(pcg::QRHO);
  const R vel[3] = {P.c(pcg::QU), P.c(pcg::QV), P.c(pcg::QW)};
  const R p = P.c(pcg::QPRES);
  const R rhoe = P.c(pcg::QREINT);
  const R enth = ((rhoe + pabs(p, p0)) / rho) / cs;
  const R alpham = R(0.5) * (dp / (rho * cc) - dvel[D]) * rho / cc;
  const R alphap = R(0.5) * (dp / (rho * cc) + dvel[D]) * rho / cc;
  const R alpha0r = drho - dp / cs;
  const R alpha0e = drhoe - dp * enth;
  const R alpha0v = dvel[l1];
  const R alpha0w = dvel[l2];
  const R wv[3] = {vel[D] - cc, vel[D], vel[D] + cc};
  {
    const R rho_ref = rho - R(0.5) * (R(1) + dtdx * dmin(wv[0], R(0))) * drho;
    R vel_ref[3];
#pragma unroll
    for (int dim = 0; dim < 3; dim++) vel_ref[dim] = vel[dim] - R(0.5) * (R(1) + dtdx * dmin(wv[0], R(0))) * dvel[dim];
    const R p_ref = p - R(0.5) * (R(1) + dtdx * dmin(wv[0], R(0))) * dp;
    const R rhoe_ref = rhoe - R(0.5) * (R(1) + dtdx * dmin(wv[0], R(0))) * drhoe;
    const R apright = R(0.25) * dtdx * (wv[0] - wv[2]) * (R(1) - copysign(R(1), wv[2])) * alphap;
    const R amright = R(0);
    const R azrright = R(0.25) * dtdx * (wv[0] - wv[1]) * (R(1) - copysign(R(1), wv[1])) * alpha0r;
    const R azeright = R(0.25) * dtdx * (wv[0] - wv[1]) * (R(1) - copysign(R(1), wv[1])) * alpha0e;
    const R azv1rght = R(0.25) * dtdx * (wv[0] - wv[1]) * (R(1) - copysign(R(1), wv[1])) * alpha0v;
    const R azw1rght = R(0.25) * dtdx * (wv[0] - wv[1]) * (R(1) - copysign(R(1), wv[1])) * alpha0w;
    R r = rho_ref + apright + amright + azrright;
    qp[pcg::TR_RHO] = dmax(Lim<R>::tiny(), r);
    qp[pcg::TR_U + D] = vel_ref[D] + (apright - amright) * cc / rho;
    qp[pcg::TR_U + l1] = vel_ref[l1] + azv1rght;
    qp[pcg::TR_U + l2] = vel_ref[l2] + azw1rght;
    r = p_ref + (apright + amright) * cs;
    qp[pcg::TR_P] = dmax(r, pfloor(Lim<R>::tiny(), p0));
    qp[pcg::TR_RE] = rhoe_ref + (apright + amright) * enth * cs + azeright;
  }
  {
    const R rho_ref = rho + R(0.5) * (R(1) - dtdx * dmax(wv[2], R(0))) * drho;
    R vel_ref[3];
#pragma unroll
    for (int dim = 0; dim < 3; dim++) vel_ref[dim] = vel[dim] + R(0.5) * (R(1) - dtdx * dmax(wv[2], R(0))) * dvel[dim];
    const R p_ref = p + R(0.5) * (R(1) - dtdx * dmax(wv[2], R(0))) * dp;
    const R rhoe_ref = rhoe + R(0.5) * (R(1) - dtdx * dmax(wv[2], R(0))) * drhoe;
    const R apleft = R(0);
    const R amleft = R(0.25) * dtdx * (wv[2] - wv[0]) * (R(1) + copysign(R(1), wv[0])) * alpham;
    const R azrleft = R(0.25) * dtdx * (wv[2] - wv[1]) * (R(1) + copysign(R(1), wv[1])) * alpha0r;
    const R azeleft = R(0.25) * dtdx * (wv[2] - wv[1]) * (R(1) + copysign(R(1), wv[1])) * alpha0e;
    const R azv1left = R(0.25) * dtdx * (wv[2] - wv[1]) * (R(1) + copysign(R(1), wv[1])) * alpha0v;
    const R azw1left = R(0.25) * dtdx * (wv[2] - wv[1]) * (R(1) + copysign(R(1), wv[1])) * alpha0w;
    R r = rho_ref + apleft + amleft + azrleft;
    qm[pcg::TR_RHO] = dmax(r, Lim<R>::tiny());
    qm[pcg::TR_U + D] = vel_ref[D] + (apleft - amleft) * cc / rho;
    qm[pcg::TR_U + l1] = vel_ref[l1] + azv1left;
    qm[pcg::TR_U + l2] = vel_ref[l2] + azw1left;
    r = p_ref + (apleft + amleft) * cs;
    qm[pcg::TR_P] = dmax(r, pfloor(Lim<R>::tiny(), p0));
    qm[pcg::TR_RE] = rhoe_ref + (apleft + amleft) * enth * cs + azeleft;
  }
  const R vel_ad = P.c(pcg::QU + D);
  const R spzerom = (vel_ad > R(0)) ? R(-1) : vel_ad * dtdx;
  const R spzerop = (vel_ad >= R(0)) ? vel_ad * dtdx : R(1);
#pragma unroll
  for (int n = 0; n < NS; n++) {
    const R slope = SLOPE(pcg::QFS + n);
    const R qc = P.c(pcg::QFS + n);
    const R acmprght = R(0.5) * (R(-1) - spzerom) * slope;
    qp[pcg::TR_Y + n] = qc + acmprght;
    const R acmpleft = R(0.5) * (R(1) - spzerop) * slope;
    qm[pcg::TR_Y + n] = qc + acmpleft;
  }
#undef SLOPE
}

template <int NS, bool MIX, int D, class R, class QP, class QM>
__device__ __forceinline__ void plm_cell(const pcg::Region& rg, int i, int j, int k, R cc, R flat, int order,
                                         double dt, const QP& qp, const QM& qm) {
  plm_cell_p<NS, MIX, D, R>(rg, Prim<R>(rg, i, j, k, D), cc, flat, order, dt, qp, qm);
}

template <int NS, bool MIX, bool EXACT, bool HYB, int D, class R, class PT>
__device__ __forceinline__ void trace_cell_p(const pcg::StageArgs& a, const pcg::Region& rg, const PT& P, int i, int j,
                                             int k) {
  const CellPtr<const R> pr = at(v4<const R>(rg.prep), i, j, k);
  const R flat = pr[0], cc = pr[1];
  const double dt = dt_of(a, rg);
  if (a.ppm_type == 1)
    trace_ppm_dir<NS, MIX, EXACT, HYB, D, R>(rg, P, i, j, k, cc, flat, dt, a.weno_scheme);
  else
    plm_cell_p<NS, MIX, D, R>(rg, P, cc, flat, a.plm_iorder, dt, at(b4<R>(rg.trp[D]), i, j, k),
                              at(b4<R>(rg.trm[D]), i + (D == 0), j + (D == 1), k + (D == 2)));
}

template <int NS, bool MIX, bool EXACT, bool HYB, int D, class R>
__device__ __forceinline__ void trace_cell(const pcg::StageArgs& a, const pcg::Region& rg, int i, int j, int k) {
  trace_cell_p<NS, MIX, EXACT, HYB, D, R>(a, rg, Prim<R>(rg, i, j, k, D), i, j, k);
}

template <int NS, bool MIX, bool EXACT, class R, int MINB>
__global__ void __launch_bounds__(128, MINB) k_trace(pcg::StageArgs a) {
  Item it;
  if (!item_of(a, it)) return;
  switch (it.variant) {
    case 0: trace_cell<NS, MIX, EXACT, false, 0, R>(a, *it.rg, it.i, it.j, it.k); break;
    case 1: trace_cell<NS, MIX, EXACT, false, 1, R>(a, *it.rg, it.i, it.j, it.k); break;
    default: trace_cell<NS, MIX, EXACT, false, 2, R>(a, *it.rg, it.i, it.j, it.k); break;
  }
}

// ------------------------------------------------------------------ TMA-staged trace
// The trace of the mixed form on full tiles of 128 cells (pcg::trace_tile_y/z), one cell
// per thread. One TMA load stages the FP32 primitive copy of the tile and its two-cell
// halo along the traced direction D (every component) in shared memory; every stencil of
// the trace then reads the tile at compile-time offsets from the cell. The tiles cover
// the largest part of grow(box,1) that they fill exactly, so no lane of a tile idles; the
// same launch traces the strips left over (narrower than a tile) one cell per thread
// from global memory (segment variants 0-2 strips, 3-5 tiles, of direction variant % 3).
// The PPM interface values of a tile (ppm_tile_edges): for each reconstructed component
// (the trace-state components but rho e, slot e_slot), along D the interfaces of every
// row of the tile, the low face of each cell and one past the last.
template <int D>
struct TileEdges {
  static constexpr int ROW = D == 0 ? pcg::kTraceTileX + 1 : pcg::kTraceTileX;  // x: 33 faces per row
  static constexpr int NROW = D == 0 ? 4 : 5;  // y, z: 5 face rows of 32
  static constexpr int PLANE = ROW * NROW;
  static constexpr int ST = D == 0 ? 1 : pcg::kTraceTileX;  // from a cell's low face to its high face
  // van Leer slopes of the cells of the tile and one more on each side along D
  static constexpr int DROW = D == 0 ? pcg::kTraceTileX + 2 : pcg::kTraceTileX;
  static constexpr int DPLANE = D == 0 ? DROW * 4 : DROW * 6;
};
__host__ __device__ constexpr int edge_slot(int tr) { return tr < pcg::TR_RE ? tr : tr - 1; }
__host__ __device__ constexpr int slot_tr(int e) { return e < pcg::TR_RE ? e : e + 1; }

template <int D>
struct PrimTile {
  static constexpr bool kEdges = true;
  static constexpr int BX = pcg::trace_box_x(D), BY = pcg::trace_box_y(D);
  static constexpr int PLANE = pcg::trace_box_cells(D);
  static constexpr int ST = D == 0 ? 1 : D == 1 ? BX : BX * BY;
  const float* p;  // component 0 of the cell in the tile
  const float* e;  // interface values: slot 0 on the cell's low face
  __device__ __forceinline__ float c(int qcomp) const { return p[tr_comp(qcomp) * PLANE]; }
  __device__ __forceinline__ void edges(int qcomp, float& sm, float& sp) const {
    const float* b = e + edge_slot(tr_comp(qcomp)) * TileEdges<D>::PLANE;
    sm = b[0];
    sp = b[TileEdges<D>::ST];
  }
  __device__ __forceinline__ void five(int qcomp, float* s) const { stencil<2>(qcomp, s); }
  template <int W>
  __device__ __forceinline__ void stencil(int qcomp, float* s) const {
    const float* b = p + tr_comp(qcomp) * PLANE;
#pragma unroll
    for (int o = -W; o <= W; ++o) s[o + W] = b[o * ST];
  }
};

// The PPM interface values of every reconstructed component of the staged tile along D,
// each formed once (the per-cell form evaluates three van Leer slopes and two interfaces
// per cell and component): the slopes of the tile's cells and of one more cell on each
// side along D, then the interfaces. ox: the x offset of the tile's first cell in the
// staged box. For x the four warps work on their own rows; for y and z the rows along D
// belong to different warps, so the block synchronises between the phases.
template <int NS, int D>
__device__ __forceinline__ void ppm_tile_edges(const float* tile, int ox, float* dsv, float* edg) {
  using P = PrimTile<D>;
  using G = TileEdges<D>;
  constexpr int NE = pcg::nt_comps(NS) - 1;
  const int lane = int(threadIdx.x) % 32, w = int(threadIdx.x) / 32;
  if constexpr (D == 0) {
    // row w; slope index m: cell x0 - 1 + m (m < 34); interface index f: low face of x0 + f
    const float* row = tile + w * P::BX + ox - 1;  // the cell x0 - 1
    float* drow = dsv + w * G::DROW;
    float* erow = edg + w * G::ROW;
#pragma unroll
    for (int e = 0; e < NE; ++e) {
      const float* q = row + slot_tr(e) * P::PLANE + lane;
      drow[e * G::DPLANE + lane] = vl_slope<float>(q[-1], q[0], q[1]);
    }
    if (lane < 2 * NE) {  // slopes 32 and 33 of every component
      const int e = lane >> 1, m = 32 + (lane & 1);
      const float* q = row + slot_tr(e) * P::PLANE + m;
      drow[e * G::DPLANE + m] = vl_slope<float>(q[-1], q[0], q[1]);
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < NE; ++e) {
      const float* q = row + slot_tr(e) * P::PLANE + lane;  // cells x0-1+lane (left), x0+lane
      const float* d = drow + e * G::DPLANE + lane;
      erow[e * G::PLANE + lane] = ppm_edge<float>(q[0], q[1], d[0], d[1]);
    }
    if (lane < NE) {  // face 32 of every component
      const float* q = row + slot_tr(lane) * P::PLANE + 32;
      const float* d = drow + lane * G::DPLANE + 32;
      erow[lane * G::PLANE + 32] = ppm_edge<float>(q[0], q[1], d[0], d[1]);
    }
    __syncwarp();
  } else {
    // slope row m: cells D0 - 1 + m (m < 6), staged row m + 1; face row f: low face of
    // D0 + f (f < 5), between staged rows f + 1 and f + 2 (D0 the tile's first y or z)
    constexpr int RS = P::ST;  // staged-row stride along D
    const float* col = tile + ox + lane;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int m = w + 4 * h;
      if (h == 0 || m < 6) {
#pragma unroll
        for (int e = 0; e < NE; ++e) {
          const float* q = col + slot_tr(e) * P::PLANE + (m + 1) * RS;
          dsv[e * G::DPLANE + m * 32 + lane] = vl_slope<float>(q[-RS], q[0], q[RS]);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int f = w + 4 * h;
      if (h == 0 || f < 5) {
#pragma unroll
        for (int e = 0; e < NE; ++e) {
          const float* q = col + slot_tr(e) * P::PLANE + (f + 1) * RS;
          const float* d = dsv + e * G::DPLANE + f * 32 + lane;
          edg[e * G::PLANE + f * 32 + lane] = ppm_edge<float>(q[0], q[RS], d[0], d[32]);
        }
      }
    }
    __syncthreads();
  }
}

template <int NS, bool MIX, int D>
__device__ __forceinline__ void trace_tile(const pcg::StageArgs& a, const pcg::Seg& sg, int t, float* tile,
                                           float* dsv, float* edg, uint64_t* bar) {
  using P = PrimTile<D>;
  constexpr int NC = pcg::nt_comps(NS), TY = pcg::trace_tile_y(D), TZ = pcg::trace_tile_z(D);
  const pcg::Region& rg = a.regions[sg.region];
  const int ntx = sg.n[0], nty = sg.n[1];
  const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
  const int x0 = sg.lo[0] + pcg::kTraceTileX * tx, y0 = sg.lo[1] + TY * ty, z0 = sg.lo[2] + TZ * tz;
  const int qx = rg.qf.b[0], qy = rg.qf.b[1], qz = rg.qf.b[2];
  int xs = (D == 0) ? x0 - 2 : x0;
  xs -= (xs - qx) & 3;  // a multiple of 4 elements from the array's first x
  const int ys = (D == 1) ? y0 - 2 : y0, zs = (D == 2) ? z0 - 2 : z0;
  if (threadIdx.x == 0) {
    const void* tmap = static_cast<const char*>(a.tmaps) + (size_t(sg.region) * 3 + D) * pcg::kTensorMapBytes;
    mbar_arrive_expect_tx(bar, P::PLANE * NC * 4);
    tma_load_4d(tile, tmap, xs - qx, ys - qy, zs - qz, 0, bar);
  }
  // every thread waits for the load; if any gave up, the whole block leaves (after a second
  // bounded wait, as the load may still land), so that the block's barriers stay uniform
  const bool landed = mbar_wait_bounded(bar, 0);
  if (__syncthreads_or(!landed)) {
    if (threadIdx.x == 0 && a.err) atomicOr(a.err, 1);
    if (!landed) mbar_wait_bounded(bar, 0);
    return;
  }
  if (a.ppm_type == 1) ppm_tile_edges<NS, D>(tile, x0 - xs, dsv, edg);
  const int lane = int(threadIdx.x) % pcg::kTraceTileX, row = int(threadIdx.x) / pcg::kTraceTileX;
  const int i = x0 + lane, j = y0 + (TY > 1 ? row : 0), k = z0 + (TZ > 1 ? row : 0);
  if (i > rg.hi[0] + 1 || j > rg.hi[1] + 1 || k > rg.hi[2] + 1) return;  // tiles lie in grow(box, 1)
  const P prim{tile + ((k - zs) * P::BY + (j - ys)) * P::BX + (i - xs), edg + row * TileEdges<D>::ROW + lane};
  trace_cell_p<NS, MIX, false, false, D, float>(a, rg, prim, i, j, k);
}

template <int NS, bool MIX, int MINB>
__global__ void __launch_bounds__(128, MINB) k_trace_tile(pcg::StageArgs a) {
  constexpr int kBoxMax = pcg::trace_box_cells(1) > pcg::trace_box_cells(2) ? pcg::trace_box_cells(1)
                                                                             : pcg::trace_box_cells(2);
  static_assert(pcg::trace_box_cells(0) <= kBoxMax, "tile buffer");
  constexpr int NE = pcg::nt_comps(NS) - 1;
  constexpr int kDsv = TileEdges<1>::DPLANE > TileEdges<0>::DPLANE ? TileEdges<1>::DPLANE : TileEdges<0>::DPLANE;
  constexpr int kEdg = TileEdges<1>::PLANE > TileEdges<0>::PLANE ? TileEdges<1>::PLANE : TileEdges<0>::PLANE;
  __shared__ __align__(128) float tile[kBoxMax * pcg::nt_comps(NS)];
  __shared__ float dsv[NE * kDsv];  // van Leer slopes (PPM)
  __shared__ float edg[NE * kEdg];  // interface values (PPM)
  __shared__ __align__(8) uint64_t bar;
  static_assert(sizeof(tile) + sizeof(dsv) + sizeof(edg) + 8 <= 48 * 1024, "tile shared memory");
  int t;
  const pcg::Seg& sg = seg_of(a, t);
  if (sg.variant < 3) {  // a strip: one cell per thread (the block's segment is uniform)
    const unsigned local = unsigned(t) * blockDim.x + threadIdx.x;
    if (local >= (unsigned)sg.count) return;
    const unsigned n0 = sg.n[0], n1 = sg.n[1];
    const unsigned r = local / n0;
    const int i = sg.lo[0] + (int)(local - r * n0), j = sg.lo[1] + (int)(r % n1), k = sg.lo[2] + (int)(r / n1);
    const pcg::Region& rg = a.regions[sg.region];
    switch (sg.variant) {
      case 0: trace_cell<NS, MIX, false, false, 0, float>(a, rg, i, j, k); break;
      case 1: trace_cell<NS, MIX, false, false, 1, float>(a, rg, i, j, k); break;
      default: trace_cell<NS, MIX, false, false, 2, float>(a, rg, i, j, k); break;
    }
    return;
  }
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  switch (sg.variant) {
    case 3: trace_tile<NS, MIX, 0>(a, sg, t, tile, dsv, edg, &bar); break;
    case 4: trace_tile<NS, MIX, 1>(a, sg, t, tile, dsv, edg, &bar); break;
    default: trace_tile<NS, MIX, 2>(a, sg, t, tile, dsv, edg, &bar); break;
  }
}

// The PPM trace with hybrid-WENO edge values (use_hybrid_weno): its own kernel, so that
// the WENO code does not weigh on the registers of the plain trace.
template <int NS, bool MIX, bool EXACT, class R>
__global__ void __launch_bounds__(128) k_trace_weno(pcg::StageArgs a) {
  Item it;
  if (!item_of(a, it)) return;
  switch (it.variant) {
    case 0: trace_cell<NS, MIX, EXACT, true, 0, R>(a, *it.rg, it.i, it.j, it.k); break;
    case 1: trace_cell<NS, MIX, EXACT, true, 1, R>(a, *it.rg, it.i, it.j, it.k); break;
    default: trace_cell<NS, MIX, EXACT, true, 2, R>(a, *it.rg, it.i, it.j, it.k); break;
  }
}

// ------------------------------------------------------------------ flux stages
template <int NS, class R, class C>
__device__ __forceinline__ void load_state(const C& t, R* s) {
#pragma unroll
  for (int n = 0; n < pcg::nt_comps(NS); ++n) s[n] = t[n];
}

// p0: the region's pressure offset of the FP32 arithmetic (p0_of), formed once by the
// caller rather than per face (it reads the FP64 state of the region's first cell).
template <int NS, bool MIX, bool EXACT, int D, class R, bool QX = false>
__device__ __forceinline__ void face_flux(const pcg::Region& rg, int i, int j, int k, const R* ql, const R* qr,
                                          R p0, R* fl, R& gun, R& gpres, R* qx = nullptr) {
  const V4<const double> qav = v4<const double>(rg.qa);
  const CellPtr<const double> qa = at(qav, i, j, k);
  const R cav = R(0.5 * (qa[pcg::QC] + qa.p[-dstride(qav, D) + pcg::QC * qa.ns]));
  const int idx = (D == 0) ? i : (D == 1) ? j : k;
  cmpflx<NS, MIX, EXACT, D, R, QX>(ql, qr, idx, rg.bclo[D], rg.bchi[D], rg.domlo[D], rg.domhi[D], cav, p0, fl, gun,
                                   gpres, qx);
}

template <int NS, class R, class C>
__device__ __forceinline__ void store_tflux(const C& f, const R* fl, R gun, R gpres) {
#pragma unroll
  for (int n = 0; n < 5; ++n) f[n] = fl[n];
#pragma unroll
  for (int n = 0; n < NS; ++n) f[pcg::FL_Y + n] = fl[pcg::UFS + n];
  f[pcg::FL_Y + NS] = gpres;
  f[pcg::FL_Y + NS + 1] = gun;
}

// First Riemann solves (Source/Godunov.cpp:206-244).
template <int NS, bool MIX, bool EXACT, int D, class R>
__device__ __forceinline__ void flux0_face(const pcg::Region& rg, int i, int j, int k) {
  R ql[pcg::nt_comps(NS)], qr[pcg::nt_comps(NS)], fl[pcg::nvar(NS)], gun, gpres;
  load_state<NS, R>(at(b4<R>(rg.trm[D]), i, j, k), ql);
  load_state<NS, R>(at(b4<R>(rg.trp[D]), i, j, k), qr);
  face_flux<NS, MIX, EXACT, D, R>(rg, i, j, k, ql, qr, R(p0_of<NS, MIX, R>(rg)), fl, gun, gpres);
  store_tflux<NS, R>(at(b4<R>(rg.fi[D]), i, j, k), fl, gun, gpres);
}

template <int NS, bool MIX, bool EXACT, class R, int MINB>
__global__ void __launch_bounds__(128, MINB) k_flux0(pcg::StageArgs a) {
  Item it;
  if (!item_of(a, it)) return;
  switch (it.variant) {
    case 0: flux0_face<NS, MIX, EXACT, 0, R>(*it.rg, it.i, it.j, it.k); break;
    case 1: flux0_face<NS, MIX, EXACT, 1, R>(*it.rg, it.i, it.j, it.k); break;
    default: flux0_face<NS, MIX, EXACT, 2, R>(*it.rg, it.i, it.j, it.k); break;
  }
}

// The march of one thread of a y- or z-face stage (k_flux1, k_flux2): threads in linear
// order over i (fastest), the row axis and the chunks of pcg::FACE_MARCH faces along D.
template <int D>
__device__ __forceinline__ bool march_of(const pcg::Seg& sg, int t, int& i, int& r, int& m0, int& m1) {
  constexpr int RA = (D == 1) ? 2 : 1;
  const unsigned local = unsigned(t) * blockDim.x + threadIdx.x;
  if (local >= (unsigned)pcg::face_threads(D, sg.n)) return false;
  const unsigned n0 = sg.n[0], nr = sg.n[RA];
  const unsigned q = local / n0;
  i = sg.lo[0] + (int)(local - q * n0);
  r = sg.lo[RA] + (int)(q % nr);
  m0 = sg.lo[D] + (int)(q / nr) * pcg::FACE_MARCH;
  m1 = min(m0 + pcg::FACE_MARCH, sg.lo[D] + sg.n[D]);
  return true;
}

// pc_transdo (Source/Godunov.H:455-633) split like pc_transdd below: transdo_corr forms
// the part that depends only on the cell the traced state belongs to, the O-flux
// differences of the conserved components and the pressure update,
//   K[n]      = cdtdx (F^O_{+} - F^O)[n],  n < 5 + NS,
//   K[5 + NS] = cdtdx (dAup + pav dAu (c - 1))   (+ p0 c dAu in the FP32 form),
// and transdo_apply corrects one traced state with it, by the reference's expressions.
template <int NS> constexpr int ncorr1() { return 6 + NS; }

// The O-correction of one cell formed on demand from its two O-fluxes (component n of K).
template <int NS, class R, class C = BCell<const R>>
struct TransdoCorr {
  C f, g;  // the cell's first O-fluxes on its low and high O-faces
  R cdtdx, c, p0;
  __device__ __forceinline__ R operator()(int n) const {
    if (n < pcg::FL_Y + NS) return cdtdx * (g[n] - f[n]);
    const R pggp = g[pcg::FL_Y + NS];
    const R pggm = f[pcg::FL_Y + NS];
    const R ugp = g[pcg::FL_Y + NS + 1];
    const R ugm = f[pcg::FL_Y + NS + 1];
    const R dAup = pggp * ugp - pggm * ugm;
    const R pav = R(0.5) * (pggp + pggm);
    const R dAu = ugp - ugm;
    R dpt = dAup + pav * dAu * (c - R(1));
    if constexpr (PDev<R>::on) dpt = dpt + p0 * c * dAu;
    return cdtdx * dpt;
  }
};
// A correction already formed (K[n]).
template <class R>
struct CorrArray {
  const R* K;
  __device__ __forceinline__ R operator()(int n) const { return K[n]; }
};

template <int NS, class R, class C>
__device__ __forceinline__ void transdo_corr(const C& f, const C& g, R cdtdx, R c, R p0, R* K) {
  const TransdoCorr<NS, R, C> kc{f, g, cdtdx, c, p0};
  constexpr int NC = pcg::FL_Y + NS;
  if constexpr (sizeof(R) == 4) {
    // the flux differences in component pairs with packed FP32 (FMUL2)
    const float2 c2 = make_float2(cdtdx, cdtdx);
#pragma unroll
    for (int m = 0; m < NC / 2; ++m) {
      const int n = 2 * m;
      const float2 v = __fmul2_rn(c2, __fadd2_rn(make_float2(g[n], g[n + 1]), make_float2(-f[n], -f[n + 1])));
      K[n] = v.x;
      K[n + 1] = v.y;
    }
    if constexpr (NC % 2) K[NC - 1] = kc(NC - 1);
    K[NC] = kc(NC);
  } else {
#pragma unroll
    for (int n = 0; n < ncorr1<NS>(); ++n) K[n] = kc(n);
  }
}

template <int NS, bool EXACT, class R, class KF>
__device__ __forceinline__ void transdo_apply(const R* qn, const KF& K, R p0, R* out) {
  const R flxrho = K(0);
  const R flxu = K(1);
  const R flxv = K(2);
  const R flxw = K(3);
  const R flxe = K(4);
  const R rr = qn[pcg::TR_RHO];
  const R rrnew = rr - flxrho;
  const R irrnew = EXACT ? R(0) : rrcp(rrnew);
  if constexpr (sizeof(R) == 4 && NS > 1) {
    R kc[NS];
#pragma unroll
    for (int n = 0; n < NS; n++) kc[n] = K(pcg::FL_Y + n);
    scale_sub2<NS>(rr, qn + pcg::TR_Y, kc, irrnew, out + pcg::TR_Y);
  } else {
#pragma unroll
    for (int n = 0; n < NS; n++) {
      const R compn = K(pcg::FL_Y + n);
      const R compo = rr * qn[pcg::TR_Y + n] - compn;
      out[pcg::TR_Y + n] = EXACT ? compo / rrnew : compo * irrnew;
    }
  }
  R ru = qn[pcg::TR_U], rv = qn[pcg::TR_V], rw = qn[pcg::TR_W];
  const R ekin = R(0.5) * rr * (ru * ru + rv * rv + rw * rw);
  ru *= rr;
  rv *= rr;
  rw *= rr;
  const R re = qn[pcg::TR_RE] + ekin;
  const R runew = ru - flxu;
  const R rvnew = rv - flxv;
  const R rwnew = rw - flxw;
  const R renew = re - flxe;
  out[pcg::TR_RHO] = rrnew;
  out[pcg::TR_U] = EXACT ? runew / rrnew : runew * irrnew;
  out[pcg::TR_V] = EXACT ? rvnew / rrnew : rvnew * irrnew;
  out[pcg::TR_W] = EXACT ? rwnew / rrnew : rwnew * irrnew;
  const R ke2 = runew * runew + rvnew * rvnew + rwnew * rwnew;
  const R rhoekin = EXACT ? R(0.5) * ke2 / rrnew : R(0.5) * ke2 * irrnew;
  out[pcg::TR_RE] = renew - rhoekin;
  const R pnew = qn[pcg::TR_P] - K(5 + NS);
  out[pcg::TR_P] = dmax(pnew, pfloor(Lim<R>::very_small(), p0));
}

// The O-correction of the cell (i, j, k): the first O-fluxes on its two O-faces and
// its gamma_c.
template <int NS, int O, class R>
__device__ __forceinline__ void flux1_corr(const pcg::Region& rg, int i, int j, int k, R cdt, R p0, R* K) {
  const B4<const R> fov = b4<const R>(rg.fi[O]);
  const R c = R(v4<const double>(rg.qa)(i, j, k, pcg::QGAMC));
  transdo_corr<NS, R>(at(fov, i, j, k), at_up(fov, i, j, k, O), cdt, c, p0, K);
}

// The (D|O) flux at the D-face (i, j, k) from the left and right O-corrections
// (Source/Godunov.cpp:246-384).
template <int NS, bool EXACT, int D, int SIDE, class R, class KF>
__device__ __forceinline__ void flux1_state_fn(const pcg::Region& rg, int i, int j, int k, const KF& K, R p0, R* q) {
  R qn[pcg::nt_comps(NS)];
  load_state<NS, R>(at(b4<R>(SIDE == 0 ? rg.trm[D] : rg.trp[D]), i, j, k), qn);
  transdo_apply<NS, EXACT, R>(qn, K, p0, q);
}
template <int NS, bool EXACT, int D, int SIDE, class R>
__device__ __forceinline__ void flux1_state(const pcg::Region& rg, int i, int j, int k, const R* K, R p0, R* q) {
  flux1_state_fn<NS, EXACT, D, SIDE, R>(rg, i, j, k, CorrArray<R>{K}, p0, q);
}

// The O-correction of the cell (i, j, k), formed on demand.
template <int NS, int O, class R>
__device__ __forceinline__ TransdoCorr<NS, R> flux1_corr_fn(const pcg::Region& rg, int i, int j, int k, R cdt, R p0) {
  const B4<const R> fov = b4<const R>(rg.fi[O]);
  return TransdoCorr<NS, R>{at(fov, i, j, k), at_up(fov, i, j, k, O), cdt,
                            R(v4<const double>(rg.qa)(i, j, k, pcg::QGAMC)), p0};
}

template <int NS, bool MIX, bool EXACT, int D, int O, class R>
__device__ __forceinline__ void flux1_riemann(const pcg::Region& rg, int i, int j, int k, const R* ql, const R* qr,
                                              R p0) {
  R fl[pcg::nvar(NS)], gun, gpres;
  face_flux<NS, MIX, EXACT, D, R>(rg, i, j, k, ql, qr, p0, fl, gun, gpres);
  store_tflux<NS, R>(at(b4<R>(rg.fdo[D][O]), i, j, k), fl, gun, gpres);
}

template <int NS, bool MIX, bool EXACT, int D, int O, class R>
__device__ __forceinline__ void flux1_solve(const pcg::Region& rg, int i, int j, int k, const R* Kl, const R* Kr,
                                            R p0) {
  R ql[pcg::nt_comps(NS)], qr[pcg::nt_comps(NS)];
  flux1_state<NS, EXACT, D, 0, R>(rg, i, j, k, Kl, p0, ql);
  flux1_state<NS, EXACT, D, 1, R>(rg, i, j, k, Kr, p0, qr);
  flux1_riemann<NS, MIX, EXACT, D, O, R>(rg, i, j, k, ql, qr, p0);
}

template <int NS, class R>
__device__ __forceinline__ R flux1_cdt(const pcg::StageArgs& a, const pcg::Region& rg, int O) {
  return R(1.0 / 3.0 * dt_of(a, rg) / rg.dx[O]);
}

// x-faces, one face per thread in linear order (i fastest): each lane forms the
// correction of the cell left of its face and reads the one right of it from the next
// lane's shared-memory slot, which holds that cell whenever it is in the same row; the
// last lane of a warp and the last face of a row form it themselves. The (0|O) flux
// exists where the face's O index lies in the box.
template <int NS, bool MIX, bool EXACT, int O, class R>
__device__ __forceinline__ void flux1_x_pair(const pcg::StageArgs& a, const pcg::Region& rg, bool active, bool own_right,
                                             int i, int j, int k, R p0, R* kx) {
  const int c[3] = {i, j, k};
  const bool has = active && c[O] >= rg.lo[O] && c[O] <= rg.hi[O];
  const R cdt = flux1_cdt<NS, R>(a, rg, O);
  R* mine = kx + threadIdx.x;
  R K[ncorr1<NS>()];
  if (has) {
    flux1_corr<NS, O, R>(rg, i - 1, j, k, cdt, p0, K);
#pragma unroll
    for (int n = 0; n < ncorr1<NS>(); ++n) mine[n * 128] = K[n];
  }
  __syncwarp();
  if (!has) return;
  R Kr[ncorr1<NS>()];
  if (own_right) {
    flux1_corr<NS, O, R>(rg, i, j, k, cdt, p0, Kr);
  } else {
#pragma unroll
    for (int n = 0; n < ncorr1<NS>(); ++n) Kr[n] = mine[n * 128 + 1];
  }
  flux1_solve<NS, MIX, EXACT, 0, O, R>(rg, i, j, k, K, Kr, p0);
}

template <int NS, bool MIX, bool EXACT, class R>
__device__ __forceinline__ void flux1_x(const pcg::StageArgs& a, const pcg::Seg& sg, int t, R* kx) {
  const pcg::Region& rg = a.regions[sg.region];
  const unsigned local = unsigned(t) * blockDim.x + threadIdx.x;
  const bool active = local < (unsigned)sg.count;
  const unsigned n0 = sg.n[0], n1 = sg.n[1];
  const unsigned q = local / n0;
  const int i = sg.lo[0] + (int)(local - q * n0);
  const int j = sg.lo[1] + (int)(q % n1);
  const int k = sg.lo[2] + (int)(q / n1);
  const bool own_right = (threadIdx.x & 31) == 31 || i == sg.lo[0] + sg.n[0] - 1;
  const R p0 = R(p0_of<NS, MIX, R>(rg));
  flux1_x_pair<NS, MIX, EXACT, 1, R>(a, rg, active, own_right, i, j, k, p0, kx);
  flux1_x_pair<NS, MIX, EXACT, 2, R>(a, rg, active, own_right, i, j, k, p0, kx + ncorr1<NS>() * 128);
}

// y- and z-faces: each thread marches pcg::FACE_MARCH faces along D (threads in linear
// order over i, the row axis and the march chunks). Per partner O the correction of
// the cell behind the face waits in the thread's shared-memory slot (component-major).
template <int NS, bool MIX, bool EXACT, int D, int O, class R>
__device__ __forceinline__ void flux1_march_pair(const pcg::Region& rg, int i, int r, int m, R cdt, R p0, R* slot) {
  const int j = (D == 1) ? m : r, k = (D == 1) ? r : m;
  R K[ncorr1<NS>()], qr[pcg::nt_comps(NS)], ql[pcg::nt_comps(NS)];
  flux1_corr<NS, O, R>(rg, i, j, k, cdt, p0, K);
  flux1_state<NS, EXACT, D, 1, R>(rg, i, j, k, K, p0, qr);
#pragma unroll
  for (int n = 0; n < ncorr1<NS>(); ++n) {
    const R kl = slot[n * 128];
    slot[n * 128] = K[n];
    K[n] = kl;
  }
  flux1_state<NS, EXACT, D, 0, R>(rg, i, j, k, K, p0, ql);
  flux1_riemann<NS, MIX, EXACT, D, O, R>(rg, i, j, k, ql, qr, p0);
}

template <int NS, bool MIX, bool EXACT, int D, class R>
__device__ __forceinline__ void flux1_march(const pcg::StageArgs& a, const pcg::Seg& sg, int t, R* kcarry) {
  const pcg::Region& rg = a.regions[sg.region];
  constexpr int RA = (D == 1) ? 2 : 1;  // row axis, also the second partner
  int i, r, m0, m1;
  if (!march_of<D>(sg, t, i, r, m0, m1)) return;
  const R p0 = R(p0_of<NS, MIX, R>(rg));
  const bool has0 = i >= rg.lo[0] && i <= rg.hi[0];     // (D|0) exists
  const bool hasr = r >= rg.lo[RA] && r <= rg.hi[RA];  // (D|RA) exists
  const R cdt0 = flux1_cdt<NS, R>(a, rg, 0), cdtr = flux1_cdt<NS, R>(a, rg, RA);
  R* s0 = kcarry + threadIdx.x;
  R* sr = kcarry + ncorr1<NS>() * 128 + threadIdx.x;
  R K[ncorr1<NS>()];
  const int jb = (D == 1) ? m0 - 1 : r, kb = (D == 1) ? r : m0 - 1;
  if (has0) {
    flux1_corr<NS, 0, R>(rg, i, jb, kb, cdt0, p0, K);
#pragma unroll
    for (int n = 0; n < ncorr1<NS>(); ++n) s0[n * 128] = K[n];
  }
  if (hasr) {
    flux1_corr<NS, RA, R>(rg, i, jb, kb, cdtr, p0, K);
#pragma unroll
    for (int n = 0; n < ncorr1<NS>(); ++n) sr[n * 128] = K[n];
  }
  for (int m = m0; m < m1; ++m) {
    if (has0) flux1_march_pair<NS, MIX, EXACT, D, 0, R>(rg, i, r, m, cdt0, p0, s0);
    if (hasr) flux1_march_pair<NS, MIX, EXACT, D, RA, R>(rg, i, r, m, cdtr, p0, sr);
  }
}

// FP64 forms: one D-face per thread, both corrections of each pair formed by the
// thread component by component as the state update consumes them (in FP64 the
// shared forms above hold more registers than they save).
template <int NS, bool MIX, bool EXACT, int D, class R>
__device__ __forceinline__ void flux1_face(const pcg::StageArgs& a, const pcg::Region& rg, int i, int j, int k) {
  constexpr int O1 = (D == 0) ? 1 : 0;
  constexpr int O2 = (D == 2) ? 1 : 2;
  const int c[3] = {i, j, k};
  const int di = (D == 0), dj = (D == 1), dk = (D == 2);
  const R p0 = R(p0_of<NS, MIX, R>(rg));
  // (D|O) exists where the face's O index lies in the box
  if (c[O1] >= rg.lo[O1] && c[O1] <= rg.hi[O1]) {
    const R cdt = flux1_cdt<NS, R>(a, rg, O1);
    R ql[pcg::nt_comps(NS)], qr[pcg::nt_comps(NS)];
    flux1_state_fn<NS, EXACT, D, 0, R>(rg, i, j, k, flux1_corr_fn<NS, O1, R>(rg, i - di, j - dj, k - dk, cdt, p0), p0,
                                    ql);
    flux1_state_fn<NS, EXACT, D, 1, R>(rg, i, j, k, flux1_corr_fn<NS, O1, R>(rg, i, j, k, cdt, p0), p0, qr);
    flux1_riemann<NS, MIX, EXACT, D, O1, R>(rg, i, j, k, ql, qr, p0);
  }
  if (c[O2] >= rg.lo[O2] && c[O2] <= rg.hi[O2]) {
    const R cdt = flux1_cdt<NS, R>(a, rg, O2);
    R ql[pcg::nt_comps(NS)], qr[pcg::nt_comps(NS)];
    flux1_state_fn<NS, EXACT, D, 0, R>(rg, i, j, k, flux1_corr_fn<NS, O2, R>(rg, i - di, j - dj, k - dk, cdt, p0), p0,
                                    ql);
    flux1_state_fn<NS, EXACT, D, 1, R>(rg, i, j, k, flux1_corr_fn<NS, O2, R>(rg, i, j, k, cdt, p0), p0, qr);
    flux1_riemann<NS, MIX, EXACT, D, O2, R>(rg, i, j, k, ql, qr, p0);
  }
}

template <int NS, bool MIX, bool EXACT, class R, int MINB>
__global__ void __launch_bounds__(128, MINB) k_flux1(pcg::StageArgs a) {
  if constexpr (pcg::flux1_shared(sizeof(R))) {
    __shared__ R kcarry[2 * ncorr1<NS>() * 128];
    int t;
    const pcg::Seg& sg = seg_of(a, t);
    switch (sg.variant) {
      case 0: flux1_x<NS, MIX, EXACT, R>(a, sg, t, kcarry); break;
      case 1: flux1_march<NS, MIX, EXACT, 1, R>(a, sg, t, kcarry); break;
      default: flux1_march<NS, MIX, EXACT, 2, R>(a, sg, t, kcarry); break;
    }
  } else {
    Item it;
    if (!item_of(a, it)) return;
    switch (it.variant) {
      case 0: flux1_face<NS, MIX, EXACT, 0, R>(a, *it.rg, it.i, it.j, it.k); break;
      case 1: flux1_face<NS, MIX, EXACT, 1, R>(a, *it.rg, it.i, it.j, it.k); break;
      default: flux1_face<NS, MIX, EXACT, 2, R>(a, *it.rg, it.i, it.j, it.k); break;
    }
  }
}

// Source/Godunov.H:639-845 (pc_transdd) for one side: fx is the O1-flux corrected by
// O2 positioned at the cell's low O1-face, fy the O2-flux corrected by O1 at the low
// O2-face.
// pc_transdd (Source/Godunov.H:639-845) split in two. transdd_corr forms the part that
// depends only on the cell the traced state belongs to: the two transverse flux
// differences of each conserved component and the two transverse pressure updates,
//   K[n]      = cdtdx0 (F^x_{+} - F^x)[n] + cdtdx1 (F^y_{+} - F^y)[n],  n < 5 + NS
//   K[5 + NS] = cdtdx0 (dAup_x + pav_x dAu_x (c - 1)),  K[6 + NS] the same in y,
// with c the cell's gamma_c (in the FP32 form both pressure updates also carry
// p0 c dAu). transdd_apply then corrects one traced state with K. The two D-faces of
// a cell share its K, so a thread computes it once for both. Every value is formed by
// the reference's expressions in the reference's order.
template <int NS> constexpr int ncorr() { return 7 + NS; }

template <int NS, class R, class C>
__device__ __forceinline__ void transdd_corr(const C& fx, const C& gx, const C& fy, const C& gy, R cdtdx0, R cdtdx1,
                                             R c, R p0, R* K) {
  constexpr int NC = pcg::FL_Y + NS;
  if constexpr (sizeof(R) == 4) {
    // component pairs with packed FP32 (FFMA2)
    const float2 c0 = make_float2(cdtdx0, cdtdx0), c1 = make_float2(cdtdx1, cdtdx1);
#pragma unroll
    for (int m = 0; m < NC / 2; ++m) {
      const int n = 2 * m;
      const float2 dx = __fadd2_rn(make_float2(gx[n], gx[n + 1]), make_float2(-fx[n], -fx[n + 1]));
      const float2 dy = __fadd2_rn(make_float2(gy[n], gy[n + 1]), make_float2(-fy[n], -fy[n + 1]));
      const float2 v = __ffma2_rn(c0, dx, __fmul2_rn(c1, dy));
      K[n] = v.x;
      K[n + 1] = v.y;
    }
    if constexpr (NC % 2) K[NC - 1] = cdtdx0 * (gx[NC - 1] - fx[NC - 1]) + cdtdx1 * (gy[NC - 1] - fy[NC - 1]);
  } else {
#pragma unroll
    for (int n = 0; n < NC; ++n) K[n] = cdtdx0 * (gx[n] - fx[n]) + cdtdx1 * (gy[n] - fy[n]);
  }
  const int gp = pcg::FL_Y + NS, gu = pcg::FL_Y + NS + 1;
  const R dAupx = gx[gp] * gx[gu] - fx[gp] * fx[gu];
  const R pavx = R(0.5) * (gx[gp] + fx[gp]);
  const R dAux = gx[gu] - fx[gu];
  const R dAupy = gy[gp] * gy[gu] - fy[gp] * fy[gu];
  const R pavy = R(0.5) * (gy[gp] + fy[gp]);
  const R dAuy = gy[gu] - fy[gu];
  R dptx = dAupx + pavx * dAux * (c - R(1));
  R dpty = dAupy + pavy * dAuy * (c - R(1));
  if constexpr (PDev<R>::on) {
    dptx = dptx + p0 * c * dAux;
    dpty = dpty + p0 * c * dAuy;
  }
  K[5 + NS] = cdtdx0 * dptx;
  K[6 + NS] = cdtdx1 * dpty;
}

template <int NS, bool EXACT, class R>
__device__ __forceinline__ void transdd_apply(const R* qn, const R* K, R hdt, bool has_src,
                                              const CellPtr<const double>& sq, R p0, R* out) {
  const R flxrho = K[0];
  const R flxu = K[1];
  const R flxv = K[2];
  const R flxw = K[3];
  const R flxe = K[4];
  const R rr = qn[pcg::TR_RHO];
  const R rrnew = rr - flxrho;
  const R irrnew = EXACT ? R(0) : rrcp(rrnew);
  if constexpr (sizeof(R) == 4 && NS > 1) {
    scale_sub2<NS>(rr, qn + pcg::TR_Y, K + pcg::FL_Y, irrnew, out + pcg::TR_Y);
    if (has_src) {
#pragma unroll
      for (int n = 0; n < NS; n++) out[pcg::TR_Y + n] += hdt * R(sq[pcg::QFS + n]);
    }
  } else {
#pragma unroll
    for (int n = 0; n < NS; n++) {
      const R srcpass = has_src ? R(sq[pcg::QFS + n]) : R(0);
      const R compn = K[pcg::FL_Y + n];
      const R compo = rr * qn[pcg::TR_Y + n] - compn;
      out[pcg::TR_Y + n] = (EXACT ? compo / rrnew : compo * irrnew) + hdt * srcpass;
    }
  }
  const R pxnew = K[5 + NS];
  const R pynew = K[6 + NS];
  const R s0 = has_src ? R(sq[pcg::QRHO]) : R(0), s1 = has_src ? R(sq[pcg::QU]) : R(0);
  const R s2 = has_src ? R(sq[pcg::QV]) : R(0), s3 = has_src ? R(sq[pcg::QW]) : R(0);
  const R s4 = has_src ? R(sq[pcg::QREINT]) : R(0), s5 = has_src ? R(sq[pcg::QPRES]) : R(0);
  const R ru = rr * qn[pcg::TR_U];
  const R rv = rr * qn[pcg::TR_V];
  const R rw = rr * qn[pcg::TR_W];
  const R ekin2 = ru * ru + rv * rv + rw * rw;
  const R ekin = EXACT ? R(0.5) * ekin2 / rr : R(0.5) * ekin2 * rrcp(rr);
  const R re = qn[pcg::TR_RE] + ekin;
  const R runew = ru - flxu;
  const R rvnew = rv - flxv;
  const R rwnew = rw - flxw;
  const R renew = re - flxe;
  out[pcg::TR_RHO] = rrnew + hdt * s0;
  out[pcg::TR_U] = (EXACT ? runew / rrnew : runew * irrnew) + hdt * s1;
  out[pcg::TR_V] = (EXACT ? rvnew / rrnew : rvnew * irrnew) + hdt * s2;
  out[pcg::TR_W] = (EXACT ? rwnew / rrnew : rwnew * irrnew) + hdt * s3;
  const R ke2 = runew * runew + rvnew * rvnew + rwnew * rwnew;
  const R rhoekin = EXACT ? R(0.5) * ke2 / rrnew : R(0.5) * ke2 * irrnew;
  out[pcg::TR_RE] = renew - rhoekin + hdt * s4;
  const R pn = qn[pcg::TR_P] - pxnew - pynew + hdt * s5;
  out[pcg::TR_P] = dmax(pn, pfloor(Lim<R>::tiny(), p0));
}

// pc_artif_visc (Source/Godunov.H:1105-1132) with the coefficient visc = dx * difmag *
// min(0, div u) already formed, then pc_norm_spec_flx (Source/Hydro.H:835-849), on the
// fluxes of one d-face; T is the flux arithmetic type. The increments are formed as
// visc * (u_i - u_{i-1}) in FP64, the reference's order of operations.
template <int NS, int D, class T>
__device__ __forceinline__ void adjust_fluxes(T* fl, const CellPtr<const double>& u, int ud, double visc,
                                              bool at_bndry) {
#pragma unroll
  for (int n = 0; n < pcg::nvar(NS); n++) {
    if (n == pcg::UTEMP) continue;
    const bool is_tang = (n == pcg::UMX || n == pcg::UMY || n == pcg::UMZ) && (n != pcg::UMX + D);
    if (!(at_bndry && is_tang)) fl[n] += T(visc * (u[n] - u.p[-ud + n * u.ns]));
  }
  fl[pcg::UTEMP] = T(0);
  T summ = T(0);
#pragma unroll
  for (int n = pcg::UFS; n < pcg::UFS + NS; ++n) summ += fl[n];
  const T fac = (summ != T(0)) ? fl[pcg::URHO] / summ : T(1);
#pragma unroll
  for (int n = pcg::UFS; n < pcg::UFS + NS; ++n) fl[n] *= fac;
}

// The transverse correction of the cell (i, j, k) for the final D-fluxes: the
// (O1|O2) and (O2|O1) fluxes on the cell's faces and the cell's gamma_c.
template <int NS, int D, class R>
__device__ __forceinline__ void flux2_corr(const pcg::Region& rg, int i, int j, int k, R cdtdx0, R cdtdx1, R p0,
                                           R* K) {
  constexpr int O1 = (D == 0) ? 1 : 0;
  constexpr int O2 = (D == 2) ? 1 : 2;
  const B4<const R> fxv = b4<const R>(rg.fdo[O1][O2]);
  const B4<const R> fyv = b4<const R>(rg.fdo[O2][O1]);
  const R c = R(v4<const double>(rg.qa)(i, j, k, pcg::QGAMC));
  transdd_corr<NS, R>(at(fxv, i, j, k), at_up(fxv, i, j, k, O1), at(fyv, i, j, k), at_up(fyv, i, j, k, O2), cdtdx0,
                      cdtdx1, c, p0, K);
}

// One traced state of the D-face (i, j, k) after pc_transdd: SIDE 0 the left state
// (trm, source terms of the cell behind the face), 1 the right state (trp).
template <int NS, bool EXACT, int D, int SIDE, class R>
__device__ __forceinline__ void flux2_state(const pcg::Region& rg, int i, int j, int k, const R* K, R hdt, R p0,
                                            R* q) {
  const bool has_src = rg.srcq.p != nullptr;
  const V4<const double> sqv = v4<const double>(rg.srcq);
  CellPtr<const double> sq = has_src ? at(sqv, i, j, k) : CellPtr<const double>{nullptr, 0};
  if (SIDE == 0 && has_src) sq = shift(sq, -dstride(sqv, D));
  R qn[pcg::nt_comps(NS)];
  load_state<NS, R>(at(b4<R>(SIDE == 0 ? rg.trm[D] : rg.trp[D]), i, j, k), qn);
  transdd_apply<NS, EXACT, R>(qn, K, hdt, has_src, sq, p0, q);
}

// Final fluxes (Source/Godunov.cpp:392-438) followed by the per-face flux adjustments
// of pc_adjust_fluxes (Source/Hydro.cpp:380-413): pc_artif_visc (Godunov.H:1067-1138),
// pc_norm_spec_flx and pc_ext_flx (Hydro.H:835-865). ql and qr are the face's traced
// states after their transverse corrections.
// pc_umeth_3D's own outputs at one final face (Source/Godunov.cpp:392-438, and the
// low-order boundary faces): the Godunov fluxes as pc_cmpflx leaves them, before
// pc_adjust_fluxes (UTEMP is not a Riemann output and is left as the caller set it), and
// the face state qint: GDU..GDW in absolute order, GDPRES and GDGAME = p / (rho e) + 1
// (Source/Riemann.H:181); GDRHO is not written (nor is it by the reference).
template <int NS, bool MIX, bool EXACT, int D, class R>
__device__ __forceinline__ void umeth_face(const pcg::Region& rg, int i, int j, int k, const R* ql, const R* qr,
                                           double p0d) {
  constexpr int t1 = (D == 0) ? 1 : 0;
  constexpr int t2 = (D == 2) ? 1 : 2;
  R flr[pcg::nvar(NS)], gun, gpres, qx[3];
  face_flux<NS, MIX, EXACT, D, R, true>(rg, i, j, k, ql, qr, R(p0d), flr, gun, gpres, qx);
  const CellPtr<double> ff = at(v4<double>(rg.ff[D]), i, j, k);
#pragma unroll
  for (int n = 0; n < pcg::nvar(NS); ++n)
    if (n != pcg::UTEMP) ff[n] = (PDev<R>::on && n == pcg::UMX + D) ? double(flr[n]) + p0d : double(flr[n]);
  const CellPtr<double> qe = at(v4<double>(rg.qec[D]), i, j, k);
  const double gp = PDev<R>::on ? double(gpres) + p0d : double(gpres);
  qe[pcg::GDU + D] = double(gun);
  qe[pcg::GDU + t1] = double(qx[0]);
  qe[pcg::GDU + t2] = double(qx[1]);
  qe[pcg::GDPRES] = gp;
  qe[pcg::GDGAME] = EXACT ? double(gpres / qx[2] + R(1)) : gp / double(qx[2]) + 1.0;
}

template <int NS, bool MIX, bool EXACT, int D, class R, bool UMETH = false>
__device__ __forceinline__ void flux2_face(const pcg::StageArgs& a, const pcg::Region& rg, int i, int j, int k,
                                           const R* ql, const R* qr, double p0d) {
  if constexpr (UMETH) {
    umeth_face<NS, MIX, EXACT, D, R>(rg, i, j, k, ql, qr, p0d);
    return;
  }
  constexpr int O1 = (D == 0) ? 1 : 0;
  constexpr int O2 = (D == 2) ? 1 : 2;
  R flr[pcg::nvar(NS)], gun, gpres;
  face_flux<NS, MIX, EXACT, D, R>(rg, i, j, k, ql, qr, R(p0d), flr, gun, gpres);
  // pc_artif_visc coefficient: difmag * min(0, average of the four nodal div u of the face)
  const V4<const double> dv = v4<const double>(rg.divu);
  const int ji = i + (O1 == 0), jj = j + (O1 == 1), jk = k + (O1 == 2);
  const int ki = i + (O2 == 0), kj = j + (O2 == 1), kk = k + (O2 == 2);
  const double div =
    a.difmag * dmin(0.0, 0.25 * (dv(i, j, k) + dv(ji, jj, jk) + dv(ki, kj, kk) +
                                 dv(ji + (O2 == 0), jj + (O2 == 1), jk + (O2 == 2))));
  const int idx = (D == 0) ? i : (D == 1) ? j : k;
  const bool at_bndry = (idx == rg.domlo[D] && rg.bclo[D] == pcg::BC_NO_SLIP_WALL) ||
                        (idx == rg.domhi[D] + 1 && rg.bchi[D] == pcg::BC_NO_SLIP_WALL);
  const double visc = rg.dx[D] * div;
  const V4<const double> uv = v4<const double>(rg.uin);
  const CellPtr<const double> u = at(uv, i, j, k);
  const int ud = dstride(uv, D);
  const double ar = rg.area[D].p ? v4<const double>(rg.area[D])(i, j, k) : rg.area_u[D];
  if constexpr (PDev<R>::on) {
    if (rg.ff_single) {
      // FP32 final fluxes for the FP64 divergence accumulation: the adjustments run in
      // FP32 on the FP32 Riemann fluxes (each viscous increment is formed in FP64 from the
      // FP64 state and rounded once); the normal momentum flux and the Godunov pressure
      // stay deviations from p0, which cancel in the divergence
      flr[pcg::UTEMP] = 0.f;
      adjust_fluxes<NS, D, float>(flr, u, ud, visc, at_bndry);
      const float arf = float(ar);
      const BCell<float> ff = at(b4<float>(rg.ff[D]), i, j, k);
#pragma unroll
      for (int n = 0; n < pcg::nvar(NS); ++n) ff[n] = flr[n] * arf;
      const BCell<float> qe = at(b4<float>(rg.qec[D]), i, j, k);
      qe[0] = float(gpres);
      qe[1] = float(gun);
      return;
    }
  }
  double fl[pcg::nvar(NS)];
#pragma unroll
  for (int n = 0; n < pcg::nvar(NS); ++n) fl[n] = (n == pcg::UTEMP) ? 0.0 : double(flr[n]);
  if constexpr (PDev<R>::on) fl[pcg::UMX + D] += p0d;  // momentum flux back to the absolute pressure
  adjust_fluxes<NS, D, double>(fl, u, ud, visc, at_bndry);
  // pc_ext_flx
  const CellPtr<double> ff = at(v4<double>(rg.ff[D]), i, j, k);
#pragma unroll
  for (int n = 0; n < pcg::nvar(NS); ++n) ff[n] = fl[n] * ar;
  const CellPtr<double> qe = at(v4<double>(rg.qec[D]), i, j, k);
  qe[0] = PDev<R>::on ? double(gpres) + p0d : double(gpres);
  qe[1] = double(gun);
}

// One launch covers the final fluxes of all three directions. The two D-faces of a cell
// share its transverse correction, so each thread forms about one correction per face:
//  * x-faces, one per thread in linear order: the correction right of a face comes from
//    the next lane's shared-memory slot (the last lane of a warp and the last face of a
//    row form it themselves);
//  * y- and z-faces: each thread marches pcg::FACE_MARCH faces along D, carrying the
//    correction of the cell behind the face.
// Block counts per segment are pcg::face_tiles on the host.
template <int NS, bool MIX, bool EXACT, class R>
__device__ __forceinline__ void flux2_consts(const pcg::StageArgs& a, const pcg::Region& rg, int D, R& cdtdx0,
                                             R& cdtdx1, R& hdt, double& p0d) {
  const int O1 = (D == 0) ? 1 : 0;
  const int O2 = (D == 2) ? 1 : 2;
  const double dt = dt_of(a, rg);
  cdtdx0 = R(0.5 * dt / rg.dx[O1]);
  cdtdx1 = R(0.5 * dt / rg.dx[O2]);
  hdt = R(0.5 * dt);
  p0d = p0_of<NS, MIX, R>(rg);
}

template <int NS, bool MIX, bool EXACT, class R, bool UMETH = false>
__device__ __forceinline__ void flux2_x(const pcg::StageArgs& a, const pcg::Seg& sg, int t, R* kx) {
  const pcg::Region& rg = a.regions[sg.region];
  const unsigned local = unsigned(t) * blockDim.x + threadIdx.x;
  const bool active = local < (unsigned)sg.count;
  const unsigned n0 = sg.n[0], n1 = sg.n[1];
  const unsigned q = local / n0;
  const int i = sg.lo[0] + (int)(local - q * n0);
  const int j = sg.lo[1] + (int)(q % n1);
  const int k = sg.lo[2] + (int)(q / n1);
  R cdtdx0, cdtdx1, hdt;
  double p0d;
  flux2_consts<NS, MIX, EXACT, R>(a, rg, 0, cdtdx0, cdtdx1, hdt, p0d);
  const R p0 = R(p0d);
  R* mine = kx + threadIdx.x;
  R K[ncorr<NS>()];
  if (active) {
    flux2_corr<NS, 0, R>(rg, i - 1, j, k, cdtdx0, cdtdx1, p0, K);
#pragma unroll
    for (int n = 0; n < ncorr<NS>(); ++n) mine[n * 128] = K[n];
  }
  __syncwarp();
  if (!active) return;
  R ql[pcg::nt_comps(NS)], qr[pcg::nt_comps(NS)];
  flux2_state<NS, EXACT, 0, 0, R>(rg, i, j, k, K, hdt, p0, ql);
  if ((threadIdx.x & 31) == 31 || i == sg.lo[0] + sg.n[0] - 1) {
    flux2_corr<NS, 0, R>(rg, i, j, k, cdtdx0, cdtdx1, p0, K);
  } else {
#pragma unroll
    for (int n = 0; n < ncorr<NS>(); ++n) K[n] = mine[n * 128 + 1];
  }
  flux2_state<NS, EXACT, 0, 1, R>(rg, i, j, k, K, hdt, p0, qr);
  flux2_face<NS, MIX, EXACT, 0, R, UMETH>(a, rg, i, j, k, ql, qr, p0d);
}

// Shared-memory correction slots of a k_flux2 thread: two (the march below) while they
// fit the 48 KB of static shared memory of a block, else one (large species counts in
// FP64), with the correction of the cell behind the face swapped through it.
template <int NS, class R>
__host__ __device__ constexpr int flux2_slots() {
  return 2 * ncorr<NS>() * 128 * int(sizeof(R)) <= 48 * 1024 ? 2 : 1;
}

template <int NS, bool MIX, bool EXACT, int D, class R, bool UMETH = false>
__device__ __forceinline__ void flux2_march(const pcg::StageArgs& a, const pcg::Seg& sg, int t, R* kcarry) {
  const pcg::Region& rg = a.regions[sg.region];
  int i, r, m0, m1;
  if (!march_of<D>(sg, t, i, r, m0, m1)) return;
  R cdtdx0, cdtdx1, hdt;
  double p0d;
  flux2_consts<NS, MIX, EXACT, R>(a, rg, D, cdtdx0, cdtdx1, hdt, p0d);
  const R p0 = R(p0d);
  if constexpr (flux2_slots<NS, R>() == 1) {
    R* sl = kcarry + threadIdx.x;
    R K[ncorr<NS>()];
    if (D == 1)
      flux2_corr<NS, D, R>(rg, i, m0 - 1, r, cdtdx0, cdtdx1, p0, K);
    else
      flux2_corr<NS, D, R>(rg, i, r, m0 - 1, cdtdx0, cdtdx1, p0, K);
#pragma unroll
    for (int n = 0; n < ncorr<NS>(); ++n) sl[n * 128] = K[n];
    for (int m = m0; m < m1; ++m) {
      const int j = (D == 1) ? m : r, k = (D == 1) ? r : m;
      flux2_corr<NS, D, R>(rg, i, j, k, cdtdx0, cdtdx1, p0, K);
      R ql[pcg::nt_comps(NS)], qr[pcg::nt_comps(NS)];
      flux2_state<NS, EXACT, D, 1, R>(rg, i, j, k, K, hdt, p0, qr);
#pragma unroll
      for (int n = 0; n < ncorr<NS>(); ++n) {
        const R kl = sl[n * 128];
        sl[n * 128] = K[n];
        K[n] = kl;
      }
      flux2_state<NS, EXACT, D, 0, R>(rg, i, j, k, K, hdt, p0, ql);
      flux2_face<NS, MIX, EXACT, D, R, UMETH>(a, rg, i, j, k, ql, qr, p0d);
    }
  } else {
  // the correction of the cell behind the face waits in one of this thread's two
  // shared-memory slots (component-major, conflict free): each step first forms the
  // correction of the next cell with nothing else live, then corrects both states
  R* sl = kcarry + threadIdx.x;
  R* sr = kcarry + ncorr<NS>() * 128 + threadIdx.x;
  R K[ncorr<NS>()];
  if (D == 1)
    flux2_corr<NS, D, R>(rg, i, m0 - 1, r, cdtdx0, cdtdx1, p0, K);
  else
    flux2_corr<NS, D, R>(rg, i, r, m0 - 1, cdtdx0, cdtdx1, p0, K);
#pragma unroll
  for (int n = 0; n < ncorr<NS>(); ++n) sl[n * 128] = K[n];
  for (int m = m0; m < m1; ++m) {
    const int j = (D == 1) ? m : r, k = (D == 1) ? r : m;
    flux2_corr<NS, D, R>(rg, i, j, k, cdtdx0, cdtdx1, p0, K);
#pragma unroll
    for (int n = 0; n < ncorr<NS>(); ++n) sr[n * 128] = K[n];
    R ql[pcg::nt_comps(NS)], qr[pcg::nt_comps(NS)];
    flux2_state<NS, EXACT, D, 1, R>(rg, i, j, k, K, hdt, p0, qr);
#pragma unroll
    for (int n = 0; n < ncorr<NS>(); ++n) K[n] = sl[n * 128];
    flux2_state<NS, EXACT, D, 0, R>(rg, i, j, k, K, hdt, p0, ql);
    R* tmp = sl;
    sl = sr;
    sr = tmp;
    flux2_face<NS, MIX, EXACT, D, R, UMETH>(a, rg, i, j, k, ql, qr, p0d);
  }
  }
}

template <int NS, bool MIX, bool EXACT, class R, int MINB, bool UMETH = false>
__global__ void __launch_bounds__(128, MINB) k_flux2(pcg::StageArgs a) {
  __shared__ R kcarry[flux2_slots<NS, R>() * ncorr<NS>() * 128];
  int t;
  const pcg::Seg& sg = seg_of(a, t);
  switch (sg.variant) {
    case 0: flux2_x<NS, MIX, EXACT, R, UMETH>(a, sg, t, kcarry); break;
    case 1: flux2_march<NS, MIX, EXACT, 1, R, UMETH>(a, sg, t, kcarry); break;
    default: flux2_march<NS, MIX, EXACT, 2, R, UMETH>(a, sg, t, kcarry); break;
  }
}

// Source/Godunov.cpp:6-55 (pc_low_order_boundary), called at :440-468 for the faces of a
// box on an inflow or user_bc domain boundary: the boundary state is given at time n, so
// the final flux there comes from PLM states of the two adjacent cells (slopes with the
// cell's flattening, the cell's qaux sound speed) without transverse corrections; the
// flux adjustments of pc_adjust_fluxes follow as for every face. Runs after K_FLUX2 and
// overwrites its results on those faces.
template <int NS, bool MIX, bool EXACT, int D, class R, bool UMETH = false>
__device__ __forceinline__ void lowbc_face(const pcg::StageArgs& a, const pcg::Region& rg, int i, int j, int k) {
  const int di = (D == 0), dj = (D == 1), dk = (D == 2);
  const double dt = dt_of(a, rg);
  const V4<const double> qav = v4<const double>(rg.qa);
  const V4<const R> prv = v4<const R>(rg.prep);
  R ql[pcg::nt_comps(NS)], qr[pcg::nt_comps(NS)], unused[pcg::nt_comps(NS)];
  // left state: the high-side state of the cell behind the face
  plm_cell<NS, MIX, D, R>(rg, i - di, j - dj, k - dk, R(qav(i - di, j - dj, k - dk, pcg::QC)),
                          prv(i - di, j - dj, k - dk, 0), a.plm_iorder, dt, RegState<R>{unused}, RegState<R>{ql});
  // right state: the low-side state of the face's own cell
  plm_cell<NS, MIX, D, R>(rg, i, j, k, R(qav(i, j, k, pcg::QC)), prv(i, j, k, 0), a.plm_iorder, dt,
                          RegState<R>{qr}, RegState<R>{unused});
  flux2_face<NS, MIX, EXACT, D, R, UMETH>(a, rg, i, j, k, ql, qr, p0_of<NS, MIX, R>(rg));
}

template <int NS, bool MIX, bool EXACT, class R, bool UMETH = false>
__global__ void __launch_bounds__(128) k_lowbc(pcg::StageArgs a) {
  Item it;
  if (!item_of(a, it)) return;
  switch (it.variant) {
    case 0: lowbc_face<NS, MIX, EXACT, 0, R, UMETH>(a, *it.rg, it.i, it.j, it.k); break;
    case 1: lowbc_face<NS, MIX, EXACT, 1, R, UMETH>(a, *it.rg, it.i, it.j, it.k); break;
    default: lowbc_face<NS, MIX, EXACT, 2, R, UMETH>(a, *it.rg, it.i, it.j, it.k); break;
  }
}

// Source/Godunov.H:1033-1060 (pc_pdivu) from pc_umeth_3D's own face states (the caller's
// NGDNV-component qec arrays of pcg_umeth), in the reference's expression order.
template <int NS>
__global__ void __launch_bounds__(128) k_pdivu(pcg::StageArgs a) {
  Item it;
  if (!item_of(a, it)) return;
  const pcg::Region& rg = *it.rg;
  const int i = it.i, j = it.j, k = it.k;
  const V4<const double> q0 = v4<const double>(rg.qec[0]), q1 = v4<const double>(rg.qec[1]),
                         q2 = v4<const double>(rg.qec[2]);
  const V4<const double> a0 = v4<const double>(rg.area[0]), a1 = v4<const double>(rg.area[1]),
                         a2 = v4<const double>(rg.area[2]);
  v4<double>(rg.pdivu)(i, j, k) =
    0.5 *
    ((q0(i + 1, j, k, pcg::GDPRES) + q0(i, j, k, pcg::GDPRES)) *
       (q0(i + 1, j, k, pcg::GDU) * a0(i + 1, j, k) - q0(i, j, k, pcg::GDU) * a0(i, j, k)) +
     (q1(i, j + 1, k, pcg::GDPRES) + q1(i, j, k, pcg::GDPRES)) *
       (q1(i, j + 1, k, pcg::GDV) * a1(i, j + 1, k) - q1(i, j, k, pcg::GDV) * a1(i, j, k)) +
     (q2(i, j, k + 1, pcg::GDPRES) + q2(i, j, k, pcg::GDPRES)) *
       (q2(i, j, k + 1, pcg::GDW) * a2(i, j, k + 1) - q2(i, j, k, pcg::GDW) * a2(i, j, k))) /
    v4<const double>(rg.vol)(i, j, k);
}

// Source/Hydro.H:14-68 (pc_srctoprim), launched over grow(bx,4) as at Source/Hydro.cpp:161-174:
// the primitive-variable sources srcQ from the conserved sources src and q, qaux. Only the
// components the reference writes are written (not QGAME, QTEMP).
template <int NS>
__global__ void __launch_bounds__(128) k_srctoprim(pcg::StageArgs a) {
  Item it;
  if (!item_of(a, it)) return;
  const pcg::Region& rg = *it.rg;
  const CellPtr<const double> q = at(v4<const double>(rg.q), it.i, it.j, it.k);
  const CellPtr<const double> qa = at(v4<const double>(rg.qa), it.i, it.j, it.k);
  const CellPtr<const double> src = at(v4<const double>(rg.src), it.i, it.j, it.k);
  const CellPtr<double> sq = at(v4<double>(rg.srcq), it.i, it.j, it.k);
  const double srcrho = src[pcg::URHO];
  const double rhoinv = 1.0 / q[pcg::QRHO];
  const double vx = q[pcg::QU];
  const double vy = q[pcg::QV];
  const double vz = q[pcg::QW];
  const double umx = src[pcg::UMX];
  const double umy = src[pcg::UMY];
  const double umz = src[pcg::UMZ];
  sq[pcg::QRHO] = srcrho;
  sq[pcg::QU] = (umx - vx * srcrho) * rhoinv;
  sq[pcg::QV] = (umy - vy * srcrho) * rhoinv;
  sq[pcg::QW] = (umz - vz * srcrho) * rhoinv;
  const double sreint = src[pcg::UEDEN] - vx * umx - vy * umy - vz * umz + srcrho * (vx * vx + vy * vy + vz * vz);
  sq[pcg::QREINT] = sreint;
  sq[pcg::QPRES] = qa[pcg::QDPDE] * (sreint - q[pcg::QREINT] * srcrho * rhoinv) * rhoinv + qa[pcg::QDPDR] * srcrho;
#pragma unroll
  for (int n = 0; n < NS; n++) sq[pcg::QFS + n] = (src[pcg::UFS + n] - q[pcg::QFS + n] * srcrho) * rhoinv;
}

// Source/Godunov.H:1033-1060 (pc_pdivu) and Source/Hydro.H:888-907 (pc_update), FP64
// accumulation. F is the element type of the final fluxes (double, or float with the
// pressure as deviation from p0; p0 cancels in the flux differences and is added back to
// the Godunov pressures of pdivu).
// The final fluxes and face states of the cell's six faces: FP64 arrays (caller's or
// workspace, Array4 layout) or the mixed form's FP32 workspace arrays (blocked layout).
template <class F> struct FinalView;
template <> struct FinalView<double> {
  using C = CellPtr<const double>;
  static __device__ __forceinline__ void cells(const pcg::View& w, int d, int i, int j, int k, C& lo, C& hi) {
    const V4<const double> v = v4<const double>(w);
    lo = at(v, i, j, k);
    hi = shift(lo, dstride(v, d));
  }
};
template <> struct FinalView<float> {
  using C = BCell<const float>;
  static __device__ __forceinline__ void cells(const pcg::View& w, int d, int i, int j, int k, C& lo, C& hi) {
    const B4<const float> v = b4<const float>(w);
    lo = at(v, i, j, k);
    hi = at_up(v, i, j, k, d);
  }
};

// The hydro source of cell (i, j, k), component by component: out(n, h_n) for n = 0 ..
// NVAR-1 (the p div u term already in h_UEINT), so that a caller can consume each
// component as it is formed instead of holding all of them.
template <int NS, class F, class OUT>
__device__ __forceinline__ void consup_each(const pcg::Region& rg, int i, int j, int k, double p0, OUT&& out) {
  using FV = FinalView<F>;
  typename FV::C f0, f0p, f1, f1p, f2, f2p, q0, q0p, q1, q1p, q2, q2p;
  FV::cells(rg.ff[0], 0, i, j, k, f0, f0p);
  FV::cells(rg.ff[1], 1, i, j, k, f1, f1p);
  FV::cells(rg.ff[2], 2, i, j, k, f2, f2p);
  FV::cells(rg.qec[0], 0, i, j, k, q0, q0p);
  FV::cells(rg.qec[1], 1, i, j, k, q1, q1p);
  FV::cells(rg.qec[2], 2, i, j, k, q2, q2p);
  const bool ua = rg.area[0].p != nullptr;
  const V4<const double> a0 = v4<const double>(rg.area[0]);
  const V4<const double> a1 = v4<const double>(rg.area[1]);
  const V4<const double> a2 = v4<const double>(rg.area[2]);
  const double a0m = ua ? a0(i, j, k) : rg.area_u[0], a0p = ua ? a0(i + 1, j, k) : rg.area_u[0];
  const double a1m = ua ? a1(i, j, k) : rg.area_u[1], a1p = ua ? a1(i, j + 1, k) : rg.area_u[1];
  const double a2m = ua ? a2(i, j, k) : rg.area_u[2], a2p = ua ? a2(i, j, k + 1) : rg.area_u[2];
  const double v = rg.vol.p ? v4<const double>(rg.vol)(i, j, k) : rg.vol_u;
  const double pdivu = 0.5 *
                       ((double(q0p[0]) + p0 + (double(q0[0]) + p0)) * (double(q0p[1]) * a0p - double(q0[1]) * a0m) +
                        (double(q1p[0]) + p0 + (double(q1[0]) + p0)) * (double(q1p[1]) * a1p - double(q1[1]) * a1m) +
                        (double(q2p[0]) + p0 + (double(q2[0]) + p0)) * (double(q2p[1]) * a2p - double(q2[1]) * a2m)) /
                       v;
  const CellPtr<double> uo = at(v4<double>(rg.uout), i, j, k);
#pragma unroll
  for (int n = 0; n < pcg::nvar(NS); ++n) {
    const double old = rg.zero_uout ? 0.0 : uo[n];
    double h = old + (double(f0[n]) - double(f0p[n]) + double(f1[n]) - double(f1p[n]) + double(f2[n]) -
                      double(f2p[n])) /
                         v;
    if (n == pcg::UEINT) h -= pdivu;
    out(n, h);
  }
}

template <int NS, class F>
__device__ __forceinline__ void consup_sum(const pcg::Region& rg, int i, int j, int k, double p0, double* h) {
  consup_each<NS, F>(rg, i, j, k, p0, [&](int n, double hn) { h[n] = hn; });
}

template <int NS, class F>
__device__ __forceinline__ void consup_cell(const pcg::Region& rg, int i, int j, int k, double p0) {
  double h[pcg::nvar(NS)];
  consup_sum<NS, F>(rg, i, j, k, p0, h);
  const CellPtr<double> uo = at(v4<double>(rg.uout), i, j, k);
#pragma unroll
  for (int n = 0; n < pcg::nvar(NS); ++n) uo[n] = h[n];
}

template <int NS, bool MIX>
__global__ void __launch_bounds__(128) k_consup(pcg::StageArgs a) {
  Item it;
  if (!item_of(a, it)) return;
  const pcg::Region& rg = *it.rg;
  if (rg.ff_single)
    consup_cell<NS, float>(rg, it.i, it.j, it.k, p0_of<NS, MIX, float>(rg));
  else
    consup_cell<NS, double>(rg, it.i, it.j, it.k, 0.0);
}

}  // namespace PCG_TU
