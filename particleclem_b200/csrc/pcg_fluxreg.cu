// pcg_fluxreg.cu -- flux register, reflux and average-down between a coarse level and
// the fine level above it: the coarse/fine use of the exported hydro fluxes.
//
// Reference: PeleC::update_flux_registers (Source/PeleC.cpp:1343-1400), called per box
// after the hydro source (Source/Hydro.cpp:281-287) with the area-weighted fluxes and the
// cell volume as "dx"; the register is reset at the start of the coarse advance
// (Source/Advance.cpp:30-31) and applied in PeleC::reflux (Source/PeleC.cpp:1403-1414)
// after the fine subcycles, from post_timestep (:1090-1092), before avgDown (:1098,
// defined at :1440). The register class itself is
// AMReX's EBFluxRegister / YAFluxRegister (not in the reference checkout); on regular
// boxes it implements the conservative refluxing of Berger & Colella (J. Comput. Phys.
// 82, 1989), restated here:
//   for a coarse cell c outside the fine region with a face f on the coarse/fine
//   boundary, s = +1 if f is c's low face and -1 if it is c's high face,
//     acc(c, f) = s * (sum over fine substeps of dt_f * sum of the fine fluxes on f)
//               - s * dt_c * (coarse flux on f)          [fluxes area-weighted]
//     reflux:   S_c += sum over c's register faces of acc(c, f) / V_c.
// The coarse contribution is CrseAdd's (-dt/dx fx(i) where the cell below is fine,
// +dt/dx fx(i+1) where the cell above is fine), the fine one FineAdd's.
//
// Layout: one register entry per coarse/fine face (the coarse cell outside, the face's
// direction and side, the fine box that owns the fine faces); entries sorted by coarse
// cell so that reflux sums a cell's entries in a fixed order (bit-reproducible). Every
// kernel is a thread per entry (or per cell); they move a few doubles per face and are
// bound by launch latency at register sizes (surfaces of fine regions), not by HBM.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pcg_hydro.h"

namespace pcg {
int set_error(int code, const char* msg);  // pcg_host.cu: pcg_last_error's message
}

namespace {

struct FrEntry {
  int32_t c[3];     // the coarse cell outside the fine region (periodic images wrapped)
  int32_t f[3];     // the fine-level index of the first fine cell on the fine side of the face
  int32_t dir;      // face direction
  int32_t sgn;      // +1: the face is c's low face, -1: c's high face
  int32_t fbox;     // fine box that owns the fine faces
  int32_t fface;    // fine-level face index along dir of those faces
};

__device__ __forceinline__ double& at(const pcg_array4& a, int i, int j, int k, int n) {
  return a.p[(i - a.begin[0]) + (j - a.begin[1]) * a.jstride + (k - a.begin[2]) * a.kstride + n * a.nstride];
}

// Coarse contribution of one coarse box: entries whose cell lies in the box [lo, hi]
// (the cell's register face is a face of the box) take -s dt F_c.
__global__ void k_crse_add(const FrEntry* e, int ne, double* acc, int nc, pcg_array4 fx, pcg_array4 fy,
                           pcg_array4 fz, int3 lo, int3 hi, double dt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ne) return;
  const FrEntry E = e[t];
  if (E.c[0] < lo.x || E.c[0] > hi.x || E.c[1] < lo.y || E.c[1] > hi.y || E.c[2] < lo.z || E.c[2] > hi.z) return;
  const pcg_array4& F = E.dir == 0 ? fx : E.dir == 1 ? fy : fz;
  int q[3] = {E.c[0], E.c[1], E.c[2]};
  if (E.sgn < 0) q[E.dir] += 1;  // c's high face
  for (int n = 0; n < nc; ++n) acc[size_t(t) * nc + n] -= double(E.sgn) * (dt * at(F, q[0], q[1], q[2], n));
}

// Fine contribution of fine box `fbox`: the entry's face covers ratio x ratio fine faces,
// summed along the second transverse direction outermost: +s dt sum F_f.
__global__ void k_fine_add(const FrEntry* e, int ne, double* acc, int nc, pcg_array4 fx, pcg_array4 fy,
                           pcg_array4 fz, int fbox, int ratio, double dt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ne) return;
  const FrEntry E = e[t];
  if (E.fbox != fbox) return;
  const pcg_array4& F = E.dir == 0 ? fx : E.dir == 1 ? fy : fz;
  const int t1 = E.dir == 0 ? 1 : 0, t2 = E.dir == 2 ? 1 : 2;
  for (int n = 0; n < nc; ++n) {
    double s = 0.0;
    for (int b = 0; b < ratio; ++b)
      for (int a = 0; a < ratio; ++a) {
        int q[3];
        q[E.dir] = E.fface;
        q[t1] = E.f[t1] + a;
        q[t2] = E.f[t2] + b;
        s += at(F, q[0], q[1], q[2], n);
      }
    acc[size_t(t) * nc + n] += double(E.sgn) * (dt * s);
  }
}

// Reflux: one thread per coarse cell with register entries, summing them in entry order.
__global__ void k_reflux(const FrEntry* e, const int32_t* cell_first, int ncell, const double* acc, int nc,
                         pcg_array4 s, double inv_vol) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncell) return;
  const int b0 = cell_first[t], b1 = cell_first[t + 1];
  const FrEntry E = e[b0];
  for (int n = 0; n < nc; ++n) {
    double v = at(s, E.c[0], E.c[1], E.c[2], n);
    for (int b = b0; b < b1; ++b) v += acc[size_t(b) * nc + n] * inv_vol;
    at(s, E.c[0], E.c[1], E.c[2], n) = v;
  }
}

// Average-down: each coarse cell of the coarsened fine box becomes the mean of its
// ratio^3 fine cells (uniform volumes), summed i fastest.
__global__ void k_avg_down(pcg_array4 fine, pcg_array4 crse, int3 clo, int3 cn, int ratio, int nc) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t ncell = int64_t(cn.x) * cn.y * cn.z;
  if (t >= ncell) return;
  const int i = clo.x + int(t % cn.x), j = clo.y + int((t / cn.x) % cn.y), k = clo.z + int(t / (int64_t(cn.x) * cn.y));
  const double w = 1.0 / double(ratio * ratio * ratio);
  for (int n = 0; n < nc; ++n) {
    double s = 0.0;
    for (int c = 0; c < ratio; ++c)
      for (int b = 0; b < ratio; ++b)
        for (int a = 0; a < ratio; ++a) s += at(fine, i * ratio + a, j * ratio + b, k * ratio + c, n);
    at(crse, i, j, k, n) = s * w;
  }
}

}  // namespace

struct pcg_fluxreg {
  int device = 0;
  int ratio = 2;
  int ncomp = 0;
  int nfine = 0;
  std::vector<int> flo, fhi;  // fine boxes, 3 ints each (fine index space)
  int ne = 0, ncell = 0;
  int clo[3] = {0, 0, 0}, chi[3] = {-1, -1, -1};  // bounding box of the register's coarse cells
  FrEntry* d_entries = nullptr;
  int32_t* d_cell_first = nullptr;
  double* d_acc = nullptr;
};

namespace {

int err(int code, const char* fmt, long long a = 0, long long b = 0) {
  char buf[256];
  snprintf(buf, sizeof(buf), fmt, a, b);
  return pcg::set_error(code, buf);
}

int cuda_err(cudaError_t e, const char* what) {
  cudaGetLastError();
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  return pcg::set_error(e == cudaErrorMemoryAllocation ? PCG_ENOMEM : PCG_ECUDA, buf);
}

int floordiv(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

bool covers_box(const pcg_array4* a, const int lo[3], const int hi[3], int nc) {
  if (!a || !a->p || a->ncomp < nc) return false;
  for (int d = 0; d < 3; ++d)
    if (lo[d] < a->begin[d] || hi[d] >= a->end[d]) return false;
  return true;
}

// The three face arrays of box [lo, hi] (d-faces lo..hi+1 along d) with nc components.
bool covers_faces(const pcg_array4* f, const int lo[3], const int hi[3], int nc) {
  if (!f) return false;
  for (int d = 0; d < 3; ++d) {
    int h[3] = {hi[0], hi[1], hi[2]};
    h[d] += 1;
    if (!covers_box(&f[d], lo, h, nc)) return false;
  }
  return true;
}

constexpr int kThreads = 128;
int blocks(int64_t n) { return int((n + kThreads - 1) / kThreads); }

// The register's device memory belongs to the device that was current at creation: a
// call made with another device current would hand that device foreign pointers.
int check_device(const pcg_fluxreg* R);

}  // namespace

namespace {
int check_device(const pcg_fluxreg* R) {
  int cur = -1;
  const cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return cuda_err(e, "fluxreg: cudaGetDevice");
  if (cur != R->device)
    return err(PCG_EINVAL, "fluxreg: the register was created on device %lld, the current device is %lld",
               R->device, cur);
  return PCG_OK;
}
}  // namespace

extern "C" {

int pcg_fluxreg_create(int32_t ncomp, const int32_t crse_domlo[3], const int32_t crse_domhi[3],
                       const int32_t periodic[3], int32_t ratio, int32_t nfine, const int32_t* fine_lo,
                       const int32_t* fine_hi, pcg_fluxreg** out) {
  if (!out || !crse_domlo || !crse_domhi || !periodic || (nfine > 0 && (!fine_lo || !fine_hi)))
    return err(PCG_EINVAL, "fluxreg: NULL argument");
  *out = nullptr;
  if (ncomp < 1) return err(PCG_EINVAL, "fluxreg: ncomp must be >= 1");
  if (ratio < 2 || ratio > 8) return err(PCG_EINVAL, "fluxreg: refinement ratio %lld outside 2..8", ratio);
  if (nfine < 0) return err(PCG_EINVAL, "fluxreg: nfine < 0");
  int dn[3];
  for (int d = 0; d < 3; ++d) {
    dn[d] = crse_domhi[d] - crse_domlo[d] + 1;
    if (dn[d] < 1) return err(PCG_EINVAL, "fluxreg: empty coarse domain");
  }
  // the coarsened fine boxes: aligned to the ratio, inside the coarse domain, disjoint
  std::vector<int> cb(6 * size_t(nfine));
  for (int b = 0; b < nfine; ++b) {
    for (int d = 0; d < 3; ++d) {
      const int lo = fine_lo[3 * b + d], hi = fine_hi[3 * b + d];
      if (hi < lo) return err(PCG_EINVAL, "fluxreg: fine box %lld is empty", b);
      if (floordiv(lo, ratio) * ratio != lo || floordiv(hi + 1, ratio) * ratio != hi + 1)
        return err(PCG_EINVAL, "fluxreg: fine box %lld is not aligned to the refinement ratio", b);
      cb[6 * b + d] = floordiv(lo, ratio);
      cb[6 * b + 3 + d] = floordiv(hi + 1, ratio) - 1;
      if (cb[6 * b + d] < crse_domlo[d] || cb[6 * b + 3 + d] > crse_domhi[d])
        return err(PCG_EINVAL, "fluxreg: fine box %lld is not inside the coarse domain", b);
    }
  }
  for (int a = 0; a < nfine; ++a)
    for (int b = a + 1; b < nfine; ++b) {
      bool overlap = true;
      for (int d = 0; d < 3; ++d)
        overlap = overlap && cb[6 * a + d] <= cb[6 * b + 3 + d] && cb[6 * b + d] <= cb[6 * a + 3 + d];
      if (overlap) return err(PCG_EINVAL, "fluxreg: fine boxes %lld and %lld overlap", a, b);
    }
  auto covered = [&](const int c[3]) {
    for (int b = 0; b < nfine; ++b) {
      bool in = true;
      for (int d = 0; d < 3; ++d) in = in && c[d] >= cb[6 * b + d] && c[d] <= cb[6 * b + 3 + d];
      if (in) return true;
    }
    return false;
  };
  std::vector<FrEntry> es;
  for (int b = 0; b < nfine; ++b)
    for (int d = 0; d < 3; ++d) {
      const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
      for (int side = 0; side < 2; ++side)
        for (int v = cb[6 * b + t2]; v <= cb[6 * b + 3 + t2]; ++v)
          for (int u = cb[6 * b + t1]; u <= cb[6 * b + 3 + t1]; ++u) {
            FrEntry E{};
            E.dir = d;
            E.fbox = b;
            E.c[t1] = u;
            E.c[t2] = v;
            // low side: the coarse cell below the box, the face is its high face
            E.c[d] = side == 0 ? cb[6 * b + d] - 1 : cb[6 * b + 3 + d] + 1;
            E.sgn = side == 0 ? -1 : +1;
            E.fface = side == 0 ? fine_lo[3 * b + d] : fine_hi[3 * b + d] + 1;
            E.f[t1] = u * ratio;
            E.f[t2] = v * ratio;
            E.f[d] = side == 0 ? fine_lo[3 * b + d] : fine_hi[3 * b + d];
            if (E.c[d] < crse_domlo[d] || E.c[d] > crse_domhi[d]) {
              if (!periodic[d]) continue;  // a domain face: no coarse cell outside
              E.c[d] += E.c[d] < crse_domlo[d] ? dn[d] : -dn[d];
            }
            if (covered(E.c)) continue;  // a face between two fine boxes
            es.push_back(E);
          }
    }
  // entries grouped by coarse cell (k, j, i order), creation order within a cell
  std::stable_sort(es.begin(), es.end(), [](const FrEntry& a, const FrEntry& b) {
    if (a.c[2] != b.c[2]) return a.c[2] < b.c[2];
    if (a.c[1] != b.c[1]) return a.c[1] < b.c[1];
    return a.c[0] < b.c[0];
  });
  std::vector<int32_t> first;
  for (size_t k = 0; k < es.size(); ++k)
    if (k == 0 || std::memcmp(es[k].c, es[k - 1].c, sizeof(es[k].c)) != 0) first.push_back(int32_t(k));
  first.push_back(int32_t(es.size()));
  pcg_fluxreg* R = new pcg_fluxreg();
  cudaGetDevice(&R->device);
  R->ratio = ratio;
  R->ncomp = ncomp;
  R->nfine = nfine;
  R->flo.assign(fine_lo, fine_lo + 3 * size_t(nfine));
  R->fhi.assign(fine_hi, fine_hi + 3 * size_t(nfine));
  R->ne = int(es.size());
  R->ncell = int(first.size()) - 1;
  for (const FrEntry& E : es)
    for (int d = 0; d < 3; ++d) {
      if (&E == &es[0] || E.c[d] < R->clo[d]) R->clo[d] = E.c[d];
      if (&E == &es[0] || E.c[d] > R->chi[d]) R->chi[d] = E.c[d];
    }
  cudaError_t e = cudaSuccess;
  if (R->ne > 0) {
    e = cudaMalloc(&R->d_entries, es.size() * sizeof(FrEntry));
    if (e == cudaSuccess) e = cudaMalloc(&R->d_cell_first, first.size() * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&R->d_acc, es.size() * size_t(ncomp) * sizeof(double));
    if (e == cudaSuccess)
      e = cudaMemcpy(R->d_entries, es.data(), es.size() * sizeof(FrEntry), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(R->d_cell_first, first.data(), first.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(R->d_acc, 0, es.size() * size_t(ncomp) * sizeof(double));
  }
  if (e != cudaSuccess) {
    pcg_fluxreg_destroy(R);
    return cuda_err(e, "fluxreg: create");
  }
  *out = R;
  return PCG_OK;
}

int pcg_fluxreg_destroy(pcg_fluxreg* R) {
  if (!R) return PCG_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(R->device);
  if (R->d_entries) cudaFree(R->d_entries);
  if (R->d_cell_first) cudaFree(R->d_cell_first);
  if (R->d_acc) cudaFree(R->d_acc);
  cudaSetDevice(cur);
  delete R;
  return PCG_OK;
}

int pcg_fluxreg_info(const pcg_fluxreg* R, int32_t* nfaces, int32_t* ncells) {
  if (!R) return err(PCG_EINVAL, "fluxreg: NULL register");
  if (nfaces) *nfaces = R->ne;
  if (ncells) *ncells = R->ncell;
  return PCG_OK;
}

int pcg_fluxreg_reset(pcg_fluxreg* R, pcg_stream_t stream) {
  if (!R) return err(PCG_EINVAL, "fluxreg: NULL register");
  if (int rc = check_device(R)) return rc;
  if (R->ne == 0) return PCG_OK;
  const cudaError_t e = cudaMemsetAsync(R->d_acc, 0, size_t(R->ne) * R->ncomp * sizeof(double),
                                        reinterpret_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? PCG_OK : cuda_err(e, "fluxreg: reset");
}

int pcg_fluxreg_crse_add(pcg_fluxreg* R, const int32_t lo[3], const int32_t hi[3], const pcg_array4* flx,
                         double dt, pcg_stream_t stream) {
  if (!R || !lo || !hi || !flx) return err(PCG_EINVAL, "fluxreg: NULL argument");
  if (int rc = check_device(R)) return rc;
  const int l[3] = {lo[0], lo[1], lo[2]}, h[3] = {hi[0], hi[1], hi[2]};
  if (h[0] < l[0] || h[1] < l[1] || h[2] < l[2]) return err(PCG_EINVAL, "fluxreg: empty coarse box");
  if (!covers_faces(flx, l, h, R->ncomp))
    return err(PCG_EINVAL, "fluxreg: the coarse fluxes must cover the box's faces with %lld components", R->ncomp);
  if (R->ne == 0) return PCG_OK;
  k_crse_add<<<blocks(R->ne), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      R->d_entries, R->ne, R->d_acc, R->ncomp, flx[0], flx[1], flx[2], make_int3(l[0], l[1], l[2]),
      make_int3(h[0], h[1], h[2]), dt);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PCG_OK : cuda_err(e, "fluxreg: crse_add");
}

int pcg_fluxreg_fine_add(pcg_fluxreg* R, const int32_t lo[3], const int32_t hi[3], const pcg_array4* flx,
                         double dt, pcg_stream_t stream) {
  if (!R || !lo || !hi || !flx) return err(PCG_EINVAL, "fluxreg: NULL argument");
  if (int rc = check_device(R)) return rc;
  int box = -1;
  for (int b = 0; b < R->nfine && box < 0; ++b)
    if (std::equal(lo, lo + 3, R->flo.begin() + 3 * b) && std::equal(hi, hi + 3, R->fhi.begin() + 3 * b)) box = b;
  if (box < 0) return err(PCG_EINVAL, "fluxreg: [lo, hi] is not one of the register's fine boxes");
  const int l[3] = {lo[0], lo[1], lo[2]}, h[3] = {hi[0], hi[1], hi[2]};
  if (!covers_faces(flx, l, h, R->ncomp))
    return err(PCG_EINVAL, "fluxreg: the fine fluxes must cover the box's faces with %lld components", R->ncomp);
  if (R->ne == 0) return PCG_OK;
  k_fine_add<<<blocks(R->ne), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      R->d_entries, R->ne, R->d_acc, R->ncomp, flx[0], flx[1], flx[2], box, R->ratio, dt);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PCG_OK : cuda_err(e, "fluxreg: fine_add");
}

int pcg_fluxreg_reflux(pcg_fluxreg* R, pcg_array4* s_crse, double vol, pcg_stream_t stream) {
  if (!R || !s_crse) return err(PCG_EINVAL, "fluxreg: NULL argument");
  if (!(vol > 0.0)) return err(PCG_EINVAL, "fluxreg: the coarse cell volume must be > 0");
  if (int rc = check_device(R)) return rc;
  if (R->ne == 0) return PCG_OK;
  if (!covers_box(s_crse, R->clo, R->chi, R->ncomp))
    return err(PCG_EINVAL, "fluxreg: the coarse state must cover the register's cells with %lld components",
               R->ncomp);
  k_reflux<<<blocks(R->ncell), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      R->d_entries, R->d_cell_first, R->ncell, R->d_acc, R->ncomp, *s_crse, 1.0 / vol);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PCG_OK : cuda_err(e, "fluxreg: reflux");
}

int pcg_average_down(const pcg_array4* fine, pcg_array4* crse, const int32_t fine_lo[3], const int32_t fine_hi[3],
                     int32_t ratio, int32_t ncomp, pcg_stream_t stream) {
  if (!fine || !crse || !fine_lo || !fine_hi) return err(PCG_EINVAL, "average_down: NULL argument");
  if (ratio < 2 || ratio > 8) return err(PCG_EINVAL, "average_down: refinement ratio %lld outside 2..8", ratio);
  if (ncomp < 1) return err(PCG_EINVAL, "average_down: ncomp must be >= 1");
  int flo[3], fhi[3], clo[3], chi[3];
  for (int d = 0; d < 3; ++d) {
    flo[d] = fine_lo[d];
    fhi[d] = fine_hi[d];
    if (fhi[d] < flo[d]) return err(PCG_EINVAL, "average_down: empty fine box");
    if (floordiv(flo[d], ratio) * ratio != flo[d] || floordiv(fhi[d] + 1, ratio) * ratio != fhi[d] + 1)
      return err(PCG_EINVAL, "average_down: the fine box is not aligned to the refinement ratio");
    clo[d] = floordiv(flo[d], ratio);
    chi[d] = floordiv(fhi[d] + 1, ratio) - 1;
  }
  if (!covers_box(fine, flo, fhi, ncomp)) return err(PCG_EINVAL, "average_down: fine state must cover the fine box");
  if (!covers_box(crse, clo, chi, ncomp)) return err(PCG_EINVAL, "average_down: coarse state must cover the box");
  const int64_t n = int64_t(chi[0] - clo[0] + 1) * (chi[1] - clo[1] + 1) * (chi[2] - clo[2] + 1);
  k_avg_down<<<blocks(n), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      *fine, *crse, make_int3(clo[0], clo[1], clo[2]),
      make_int3(chi[0] - clo[0] + 1, chi[1] - clo[1] + 1, chi[2] - clo[2] + 1), ratio, ncomp);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PCG_OK : cuda_err(e, "average_down");
}

}  // extern "C"
