// pcg_aux_kernels.cuh -- the steps either side of the advance: the CFL timestep
// reduction, the state update with the temperature Newton solve, and the single-level
// ghost fill. All FP64.
#pragma once

#include "pcg_kernels.cuh"

namespace PCG_TU {

enum { AUX_ESTDT = 0, AUX_ESTDT_FINAL, AUX_UPDATE, AUX_FILL, AUX_FILL_BOXES, AUX_ESTDT_BOXES, AUX_COPY };

__device__ __forceinline__ bool aux_item(const pcg::AuxArgs& a, const pcg::AuxBox*& bx, int& i, int& j, int& k) {
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
  i = s.lo[0] + (int)(local - t * n0);
  j = s.lo[1] + (int)(t % n1);
  k = s.lo[2] + (int)(t / n1);
  bx = a.boxes + s.region;
  return true;
}

// Block minimum with warp shuffles (blockDim.x == 128).
__device__ __forceinline__ double block_min(double v) {
  __shared__ double sh[4];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = (threadIdx.x < 4) ? sh[threadIdx.x] : DBL_MAX;
#pragma unroll
    for (int o = 2; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

// Source/Timestep.H:51-88 (pc_estdt_hydro) for one cell of state s:
// min over d of dx_d / (c + |u_d|), c from the stored temperature.
template <int NS, bool MIX>
__device__ __forceinline__ double cfl_dt(const double* s, const double* dx) {
  using E = Eos<NS, MIX, double>;
  const double rho = s[pcg::URHO];
  const double rhoInv = 1.0 / rho;
  const double T = s[pcg::UTEMP];
  double y[NS];
#pragma unroll
  for (int n = 0; n < NS; ++n) y[n] = s[pcg::UFS + n] * rhoInv;
  const double c = E::rty2cs(rho, T, y);
  double dt = DBL_MAX;
  const double ux = s[pcg::UMX] * rhoInv;
  dt = dmin(dt, dx[0] / (c + fabs(ux)));
  const double uy = s[pcg::UMY] * rhoInv;
  dt = dmin(dt, dx[1] / (c + fabs(uy)));
  const double uz = s[pcg::UMZ] * rhoInv;
  dt = dmin(dt, dx[2] / (c + fabs(uz)));
  return dt;
}

// Per-cell CFL constraints of every valid cell, block minima.
template <int NS, bool MIX>
__global__ void __launch_bounds__(128) k_estdt(pcg::AuxArgs a) {
  const pcg::AuxBox* bx;
  int i, j, k;
  double dt = DBL_MAX;
  if (aux_item(a, bx, i, j, k)) {
    const V4<const double> u = v4<const double>(bx->uin);
    double s[pcg::nvar(NS)];
#pragma unroll
    for (int n = 0; n < pcg::nvar(NS); ++n) s[n] = u(i, j, k, n);
    dt = cfl_dt<NS, MIX>(s, bx->dx);
  }
  dt = block_min(dt);
  if (threadIdx.x == 0) a.partial[blockIdx.x] = dt;
}

// Final reduction of the block minima, then estdt_hydro *= cfl (Source/PeleC.cpp:930).
__global__ void __launch_bounds__(128) k_estdt_final(pcg::AuxArgs a) {
  double v = DBL_MAX;
  for (int64_t b = threadIdx.x; b < a.npartial; b += blockDim.x) v = dmin(v, a.partial[b]);
  v = block_min(v);
  if (threadIdx.x == 0) *a.dt_out = v * a.cfl;
}

// Source/Advance.cpp:397-417 (construct_Snew, hydro only) then Source/PeleC.cpp:2289-2305
// (computeTemp): pc_rst_int_e default branch (PeleCUtilities.H:227-235) and pc_cmpTemp
// (PeleCUtilities.H:70-84), on one cell: s holds S_old on entry and S_new on exit.
// construct_Snew's pc_rst_int_e and computeTemp on the state s (already S_old + dt *
// hydro source).
template <int NS, bool MIX>
__device__ __forceinline__ void finish_cell(double* s) {
  using E = Eos<NS, MIX, double>;
  const double rho = s[pcg::URHO];
  const double rhoInv = 1.0 / rho;
  const double Up = s[pcg::UMX] * rhoInv;
  const double Vp = s[pcg::UMY] * rhoInv;
  const double Wp = s[pcg::UMZ] * rhoInv;
  const double ke = 0.5 * (Up * Up + Vp * Vp + Wp * Wp) - 0.5 * 0.0 * 0.0 * 0.0 * 0.0;
  s[pcg::UEINT] = s[pcg::UEDEN] - rho * ke;
  const double rhoInv2 = 1.0 / s[pcg::URHO];
  const double e = s[pcg::UEINT] * rhoInv2;
  double y[NS];
#pragma unroll
  for (int n = 0; n < NS; ++n) y[n] = s[pcg::UFS + n] * rhoInv2;
  s[pcg::UTEMP] = E::rey2t(e, y, s[pcg::UTEMP]);
}

template <int NS, bool MIX>
__device__ __forceinline__ void update_cell(double* s, const double* hsrc, double dt) {
#pragma unroll
  for (int n = 0; n < pcg::nvar(NS); ++n) s[n] += dt * hsrc[n];
  finish_cell<NS, MIX>(s);
}

template <int NS, bool MIX>
__global__ void __launch_bounds__(128) k_update(pcg::AuxArgs a) {
  const pcg::AuxBox* bx;
  int i, j, k;
  if (!aux_item(a, bx, i, j, k)) return;
  const double dt = a.dt_in ? *a.dt_in : bx->dt;
  const V4<const double> so = v4<const double>(bx->uin);
  const V4<const double> hs = v4<const double>(bx->uout);
  const V4<double> sn = v4<double>(bx->snew);
  double s[pcg::nvar(NS)], h[pcg::nvar(NS)];
#pragma unroll
  for (int n = 0; n < pcg::nvar(NS); ++n) {
    s[n] = so(i, j, k, n);
    h[n] = hs(i, j, k, n);
  }
  update_cell<NS, MIX>(s, h, dt);
#pragma unroll
  for (int n = 0; n < pcg::nvar(NS); ++n) sn(i, j, k, n) = s[n];
}

// The tail of a level step in one pass over the cells of each region: the flux
// divergence and p div u of pc_consup (kept in registers, the hydro source array is not
// written), S_new = S_old + dt * hydro_source with computeTemp written over the state in
// place, and the CFL constraint of S_new for the next step (block minima; the final
// minimum is k_estdt_final). Each value is formed by the same expressions as k_consup,
// k_update and k_estdt, so the step is the unfused step's.
template <int NS, bool MIX, int MINB>
__global__ void __launch_bounds__(128, MINB) k_advance(pcg::StageArgs a) {
  Item it;
  double dtc = DBL_MAX;
  if (item_of(a, it)) {
    const pcg::Region& rg = *it.rg;
    double s[pcg::nvar(NS)];
    const CellPtr<double> u = at(v4<double>(rg.uin), it.i, it.j, it.k);
    const double dt = dt_of(a, rg);
    // S_old + dt * hydro source, each component as its source is formed (the source
    // itself is never held whole)
    const auto add = [&](int n, double hn) { s[n] = u[n] + dt * hn; };
    if (rg.ff_single)
      consup_each<NS, float>(rg, it.i, it.j, it.k, p0_of<NS, MIX, float>(rg), add);
    else
      consup_each<NS, double>(rg, it.i, it.j, it.k, 0.0, add);
    finish_cell<NS, MIX>(s);
#pragma unroll
    for (int n = 0; n < pcg::nvar(NS); ++n) u[n] = s[n];
    dtc = cfl_dt<NS, MIX>(s, rg.dx);
  }
  dtc = block_min(dtc);
  if (threadIdx.x == 0) a.partial[blockIdx.x] = dtc;
}

// Single-level FillBoundary of a domain FAB that covers grow(domain, ng), every ghost
// cell in one pass. Filling the directions x, y, z in turn, each over the full extent of
// the others (periodic wrap or foextrap, the zero-gradient copy of the nearest valid
// layer), leaves in ghost cell (i, j, k) the valid cell (m_x(i), m_y(j), m_z(k)), with m_d
// the wrap or clamp of direction d and the identity on valid indices; each thread copies
// that cell directly. Threads cover the z ghost slabs (full x, y extent), then the y ghost
// slabs of the valid k, then the x ghost slabs of the valid (j, k), i fastest.
__device__ __forceinline__ int ghost_src(int c, int lo, int hi, bool periodic) {
  const int n = hi - lo + 1;
  if (c < lo) return periodic ? c + n : lo;
  if (c > hi) return periodic ? c - n : hi;
  return c;
}
// Ghost cell number t of the domain [dlo, dhi] grown by ng (t < the ghost-cell count) gets
// its value from the valid cell the fill maps it to; false when t is past the last ghost.
__device__ __forceinline__ bool fill_ghost(int64_t t, const int* dlo, const int* dhi, int ng, int periodic,
                                          const pcg::View& state, int ncomp) {
  const int n0 = dhi[0] - dlo[0] + 1, n1 = dhi[1] - dlo[1] + 1, n2 = dhi[2] - dlo[2] + 1;
  const int64_t e0 = n0 + 2 * ng, e1 = n1 + 2 * ng;
  const int64_t cz = e0 * e1 * 2 * ng, cy = e0 * 2 * ng * n2, cx = (int64_t)2 * ng * n1 * n2;
  int c[3];
  if (t < cz) {  // z ghost slabs: (i, j) over the grown extent, 2 ng layers
    const int g = (int)(t / (e0 * e1));
    c[0] = (int)(t % e0) + dlo[0] - ng;
    c[1] = (int)((t / e0) % e1) + dlo[1] - ng;
    c[2] = (g < ng) ? dlo[2] - ng + g : dhi[2] + 1 + (g - ng);
  } else if (t < cz + cy) {  // y ghost slabs of the valid k
    const int64_t u = t - cz;
    const int g = (int)((u / e0) % (2 * ng));
    c[0] = (int)(u % e0) + dlo[0] - ng;
    c[1] = (g < ng) ? dlo[1] - ng + g : dhi[1] + 1 + (g - ng);
    c[2] = (int)(u / (e0 * 2 * ng)) + dlo[2];
  } else if (t < cz + cy + cx) {  // x ghost slabs of the valid (j, k)
    const int64_t u = t - cz - cy;
    const int g = (int)(u % (2 * ng));
    c[0] = (g < ng) ? dlo[0] - ng + g : dhi[0] + 1 + (g - ng);
    c[1] = (int)((u / (2 * ng)) % n1) + dlo[1];
    c[2] = (int)(u / ((int64_t)2 * ng * n1)) + dlo[2];
  } else {
    return false;
  }
  int src[3];
  for (int d = 0; d < 3; ++d) src[d] = ghost_src(c[d], dlo[d], dhi[d], (periodic >> d) & 1);
  const V4<double> s = v4<double>(state);
  for (int comp = 0; comp < ncomp; ++comp) s(c[0], c[1], c[2], comp) = s(src[0], src[1], src[2], comp);
  return true;
}

// The ghost cells of many independent boxes (each its own domain) in one launch: the
// block finds its box by binary search over the boxes' first blocks.
__global__ void __launch_bounds__(128) k_fill_boxes(pcg::AuxArgs a) {
  const int64_t blk = blockIdx.x;
  int lo = 0, hi = a.nfill - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.fills[mid].blk0 <= blk) lo = mid; else hi = mid - 1;
  }
  const pcg::FillBox& f = a.fills[lo];
  const int64_t t = (blk - f.blk0) * blockDim.x + threadIdx.x;
  if (t >= f.count) return;
  fill_ghost(t, f.dlo, f.dhi, a.ng, f.periodic, f.state, a.ncomp);
}

// The next timestep of every box of a batched step: block b reduces the CFL minima the
// fused tail left for region b (the blocks of its advance segment), times cfl, into
// dt_boxes[b].
__global__ void __launch_bounds__(128) k_estdt_boxes(pcg::AuxArgs a) {
  const pcg::Seg& sg = a.bsegs[blockIdx.x];
  const int64_t nb = (sg.count + 127) / 128;
  double v = DBL_MAX;
  for (int64_t b = threadIdx.x; b < nb; b += blockDim.x) v = dmin(v, a.partial[sg.blk0 + b]);
  v = block_min(v);
  if (threadIdx.x == 0) a.dt_boxes[blockIdx.x] = v * a.cfl;
}

// Copy of the cells [dlo, dhi] of every component from one device FAB (state) to another
// (dst), FP64: the packing and unpacking of halo planes. One thread per cell and component.
__global__ void __launch_bounds__(128) k_copy_box(pcg::AuxArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n0 = a.dhi[0] - a.dlo[0] + 1, n1 = a.dhi[1] - a.dlo[1] + 1, n2 = a.dhi[2] - a.dlo[2] + 1;
  const int64_t cells = n0 * n1 * n2;
  if (t >= cells * a.ncomp) return;
  const int comp = (int)(t / cells);
  const int64_t c = t - comp * cells;
  const int i = a.dlo[0] + (int)(c % n0), j = a.dlo[1] + (int)((c / n0) % n1), k = a.dlo[2] + (int)(c / (n0 * n1));
  v4<double>(a.dst)(i, j, k, comp) = v4<const double>(a.state)(i, j, k, comp);
}

__global__ void __launch_bounds__(128) k_fill(pcg::AuxArgs a) {
  fill_ghost((int64_t)blockIdx.x * blockDim.x + threadIdx.x, a.dlo, a.dhi, a.ng, a.periodic, a.state, a.ncomp);
}

template <int NS, bool MIX>
static cudaError_t launch_advance_t(const pcg::StageArgs& a, int64_t nblocks, int variant, cudaStream_t s) {
  if (nblocks <= 0) return cudaSuccess;
  const dim3 grid((unsigned)nblocks), block(128);
  switch (variant) {
    case 0: k_advance<NS, MIX, kMinBlocks[K_CONSUP][0]><<<grid, block, 0, s>>>(a); break;
    case 1: k_advance<NS, MIX, kMinBlocks[K_CONSUP][1]><<<grid, block, 0, s>>>(a); break;
    case 2: k_advance<NS, MIX, kMinBlocks[K_CONSUP][2]><<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int NS, bool MIX>
static cudaError_t launch_aux_t(int which, const pcg::AuxArgs& a, int64_t nblocks, cudaStream_t s) {
  if (nblocks <= 0) return cudaSuccess;
  const dim3 grid((unsigned)nblocks), block(128);
  switch (which) {
    case AUX_ESTDT: k_estdt<NS, MIX><<<grid, block, 0, s>>>(a); break;
    case AUX_ESTDT_FINAL: k_estdt_final<<<1, block, 0, s>>>(a); break;
    case AUX_UPDATE: k_update<NS, MIX><<<grid, block, 0, s>>>(a); break;
    case AUX_FILL: k_fill<<<grid, block, 0, s>>>(a); break;
    case AUX_FILL_BOXES: k_fill_boxes<<<grid, block, 0, s>>>(a); break;
    case AUX_ESTDT_BOXES: k_estdt_boxes<<<grid, block, 0, s>>>(a); break;
    case AUX_COPY: k_copy_box<<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace PCG_TU
