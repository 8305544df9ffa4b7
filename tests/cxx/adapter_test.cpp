// adapter_test.cpp -- the body of PeleC's construct_hydro_source box loop
// (Source/Hydro.cpp:70-249, one regular box) written against the AMReX Array4 API, with
// pc_ctoprim, pc_srctoprim and pc_umdrv replaced by the library through
// include/pcg_pelec_adapter.H, on device memory. It compiles against the repository's
// AMReX-API shim (oracle/ref/shim) in place of AMReX, so the adapter a PeleC maintainer
// adds is exercised from C++ rather than from Python.
//
// usage: adapter_test <input.bin> <output.bin>
//   input : int32 nspec, ppm_type, plm_iorder, lo[3], hi[3]; float64 dx[3], dt, difmag;
//           the EOS (gamma law: gamma, mw; mixture: mw[ns], tmid[ns], a_lo[7 ns], a_hi[7 ns]);
//           the conserved state on grow(box,4) (NVAR components, Array4 order);
//           the conserved sources on grow(box,4) (NVAR components)
//   output: hydro_source on the box, then flx[0..2] on the box's faces (NVAR components)
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "pcg_amrex_shim.H"
#include "pcg_pelec_adapter.H"

namespace {

int fail(const char* what, int rc) {
  std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, pcg_last_error());
  return 1;
}

// A device FAB over box b with nc components, addressed as amrex::Array4.
struct DevFab {
  amrex::Box box;
  int nc = 0;
  double* d = nullptr;
  size_t n() const { return size_t(box.numPts()) * nc; }
  DevFab(const amrex::Box& b, int ncomp) : box(b), nc(ncomp) {
    cudaMalloc(&d, n() * sizeof(double));
    cudaMemset(d, 0, n() * sizeof(double));
  }
  ~DevFab() { cudaFree(d); }
  amrex::Array4<amrex::Real> array() const {
    return amrex::Array4<amrex::Real>(d, amrex::Dim3{box.smallEnd(0), box.smallEnd(1), box.smallEnd(2)},
                                      amrex::Dim3{box.bigEnd(0) + 1, box.bigEnd(1) + 1, box.bigEnd(2) + 1}, nc);
  }
  amrex::Array4<const amrex::Real> const_array() const { return array(); }
  void upload(const double* h) { cudaMemcpy(d, h, n() * sizeof(double), cudaMemcpyHostToDevice); }
  void download(std::vector<double>& h) const {
    h.resize(n());
    cudaMemcpy(h.data(), d, n() * sizeof(double), cudaMemcpyDeviceToHost);
  }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
    return 2;
  }
  std::FILE* fi = std::fopen(argv[1], "rb");
  if (!fi) return 2;
  int32_t hdr[9];
  double dd[5];
  if (std::fread(hdr, sizeof(int32_t), 9, fi) != 9 || std::fread(dd, sizeof(double), 5, fi) != 5) return 2;
  const int ns = hdr[0], ppm_type = hdr[1], plm_iorder = hdr[2];
  const amrex::Box bx(amrex::IntVect(hdr[3], hdr[4], hdr[5]), amrex::IntVect(hdr[6], hdr[7], hdr[8]));
  const amrex::GpuArray<amrex::Real, 3> dx{{dd[0], dd[1], dd[2]}};
  const double dt = dd[3], difmag = dd[4];
  const int nvar = 7 + ns, qvar = 8 + ns;
  int rc;
  if (ns == 1) {
    double g[2];
    if (std::fread(g, sizeof(double), 2, fi) != 2) return 2;
    if ((rc = pcg_set_eos_gamma(g[0], g[1]))) return fail("pcg_set_eos_gamma", rc);
  } else {
    std::vector<double> mw(ns), tmid(ns), alo(7 * ns), ahi(7 * ns);
    if (std::fread(mw.data(), sizeof(double), ns, fi) != size_t(ns) ||
        std::fread(tmid.data(), sizeof(double), ns, fi) != size_t(ns) ||
        std::fread(alo.data(), sizeof(double), 7 * ns, fi) != size_t(7 * ns) ||
        std::fread(ahi.data(), sizeof(double), 7 * ns, fi) != size_t(7 * ns))
      return 2;
    if ((rc = pcg_set_eos_nasa7(ns, mw.data(), tmid.data(), alo.data(), ahi.data())))
      return fail("pcg_set_eos_nasa7", rc);
  }
  const amrex::Box qbx = amrex::grow(bx, 4);
  DevFab S(qbx, nvar), src(qbx, nvar);
  {
    std::vector<double> h(S.n());
    if (std::fread(h.data(), sizeof(double), h.size(), fi) != h.size()) return 2;
    S.upload(h.data());
    if (std::fread(h.data(), sizeof(double), h.size(), fi) != h.size()) return 2;
    src.upload(h.data());
  }
  std::fclose(fi);

  // the box domain is the whole of space here: no physical boundary faces
  const int big = 1 << 30;
  const int domlo[3] = {-big, -big, -big}, domhi[3] = {big, big, big}, bc[3] = {0, 0, 0};
  cudaStream_t stream;
  cudaStreamCreate(&stream);
  const pcg_stream_t ps = reinterpret_cast<pcg_stream_t>(stream);
  const pcg_hydro_params prm = pcg_pelec::params(dx, dt, domlo, domhi, bc, bc, ppm_type, plm_iorder, true, false,
                                                 1, difmag, ns);

  // Source/Hydro.cpp:84-116: q, qaux on grow(bx,4) and pc_ctoprim
  DevFab q(qbx, qvar), qaux(qbx, 6 /* NQAUX */), srcq(qbx, qvar);
  const int32_t qlo[3] = {qbx.smallEnd(0), qbx.smallEnd(1), qbx.smallEnd(2)};
  const int32_t qhi[3] = {qbx.bigEnd(0), qbx.bigEnd(1), qbx.bigEnd(2)};
  {
    const pcg_array4 u = pcg_pelec::to_array4(S.const_array());
    pcg_array4 qq = pcg_pelec::to_array4(q.array()), qa = pcg_pelec::to_array4(qaux.array());
    if ((rc = pcg_ctoprim(&prm, qlo, qhi, &u, &qq, &qa, ps))) return fail("pcg_ctoprim", rc);
  }
  // Source/Hydro.cpp:161-174: pc_srctoprim of sources_for_hydro
  {
    const pcg_array4 qq = pcg_pelec::to_array4(q.const_array()), qa = pcg_pelec::to_array4(qaux.const_array()),
                     sr = pcg_pelec::to_array4(src.const_array());
    pcg_array4 sq = pcg_pelec::to_array4(srcq.array());
    if ((rc = pcg_srctoprim(&prm, qlo, qhi, &qq, &qa, &sr, &sq, ps))) return fail("pcg_srctoprim", rc);
  }
  // Source/Hydro.cpp:47, :84-97: hydro_source zeroed, flux FABs zeroed, geometry
  DevFab hsrc(bx, nvar), vol(bx, 1);
  std::vector<DevFab*> flx, area;
  for (int d = 0; d < 3; ++d) {
    flx.push_back(new DevFab(amrex::surroundingNodes(bx, d), nvar));
    area.push_back(new DevFab(amrex::surroundingNodes(bx, d), 1));
    std::vector<double> a(area[d]->n(), dx[(d + 1) % 3] * dx[(d + 2) % 3]);
    area[d]->upload(a.data());
  }
  {
    std::vector<double> v(vol.n(), dx[0] * dx[1] * dx[2]);
    vol.upload(v.data());
  }
  // Source/Hydro.cpp:245-249: pc_umdrv -> pcg_umdrv through the adapter
  const amrex::Array4<amrex::Real> flx_arr[3] = {flx[0]->array(), flx[1]->array(), flx[2]->array()};
  const amrex::Array4<const amrex::Real> a_arr[3] = {area[0]->const_array(), area[1]->const_array(),
                                                      area[2]->const_array()};
  rc = pcg_pelec::umdrv(bx, domlo, domhi, bc, bc, S.const_array(), hsrc.array(), q.const_array(),
                        qaux.const_array(), srcq.const_array(), dx, dt, ppm_type, plm_iorder, true, false, 1, difmag,
                        flx_arr, a_arr, vol.array(), ns, ps);
  if (rc) return fail("pcg_umdrv", rc);
  if (cudaStreamSynchronize(stream) != cudaSuccess) return fail("stream", -2);

  std::FILE* fo = std::fopen(argv[2], "wb");
  if (!fo) return 2;
  std::vector<double> h;
  hsrc.download(h);
  std::fwrite(h.data(), sizeof(double), h.size(), fo);
  for (int d = 0; d < 3; ++d) {
    flx[d]->download(h);
    std::fwrite(h.data(), sizeof(double), h.size(), fo);
    delete flx[d];
    delete area[d];
  }
  std::fclose(fo);
  cudaStreamDestroy(stream);
  std::printf("adapter_test ok\n");
  return 0;
}
