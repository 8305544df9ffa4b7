// fluxreg_test.cpp -- PeleC's refluxing of one coarse step written against the AMReX Array4
// API, with update_flux_registers (Source/PeleC.cpp:1343-1400, called from
// Source/Hydro.cpp:281-287) and reflux (Source/PeleC.cpp:1403-1414) done by the library
// through include/pcg_pelec_adapter.H, on device memory. Compiled against the
// repository's AMReX-API shim (oracle/ref/shim) in place of AMReX.
//
// usage: fluxreg_test <input.bin> <output.bin>
//   input : int32 ncomp, ratio, n (coarse domain [0, n)^3, one coarse box), nsub (fine
//           substeps), flo[3], fhi[3] (one fine box, fine index space), periodic[3];
//           float64 dt_crse, dt_fine, vol_crse;
//           the coarse box's three face FABs (ncomp components, Array4 order, d-faces
//           [0, n] along d); for each fine substep the fine box's three face FABs;
//           the coarse state on [0, n)^3 (ncomp components)
//   output: the coarse state after reflux
#include <cuda_runtime.h>

#include <cstdio>
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
  DevFab(const amrex::Box& b, int ncomp) : box(b), nc(ncomp) { cudaMalloc(&d, n() * sizeof(double)); }
  DevFab(const DevFab&) = delete;
  DevFab(DevFab&& o) noexcept : box(o.box), nc(o.nc), d(o.d) { o.d = nullptr; }
  ~DevFab() {
    if (d) cudaFree(d);
  }
  amrex::Array4<amrex::Real> array() const {
    return amrex::Array4<amrex::Real>(d, amrex::Dim3{box.smallEnd(0), box.smallEnd(1), box.smallEnd(2)},
                                      amrex::Dim3{box.bigEnd(0) + 1, box.bigEnd(1) + 1, box.bigEnd(2) + 1}, nc);
  }
  bool read(std::FILE* f) {
    std::vector<double> h(n());
    if (std::fread(h.data(), sizeof(double), n(), f) != n()) return false;
    return cudaMemcpy(d, h.data(), n() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess;
  }
};

// The three face FABs of box b (d-faces lo..hi+1 along d), read from f.
bool read_faces(std::FILE* f, const amrex::Box& b, int nc, std::vector<DevFab>& out) {
  out.clear();
  for (int d = 0; d < 3; ++d) {
    out.emplace_back(amrex::surroundingNodes(b, d), nc);
    if (!out.back().read(f)) return false;
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
    return 2;
  }
  std::FILE* fi = std::fopen(argv[1], "rb");
  if (!fi) return 2;
  int32_t h[13];
  double dd[3];
  if (std::fread(h, sizeof(int32_t), 13, fi) != 13 || std::fread(dd, sizeof(double), 3, fi) != 3) return 2;
  const int nc = h[0], ratio = h[1], n = h[2], nsub = h[3];
  const int32_t flo[3] = {h[4], h[5], h[6]}, fhi[3] = {h[7], h[8], h[9]}, periodic[3] = {h[10], h[11], h[12]};
  const double dt_c = dd[0], dt_f = dd[1], vol = dd[2];
  const amrex::Box cbox(amrex::IntVect(0, 0, 0), amrex::IntVect(n - 1, n - 1, n - 1));
  const amrex::Box fbox(amrex::IntVect(flo[0], flo[1], flo[2]), amrex::IntVect(fhi[0], fhi[1], fhi[2]));
  const int32_t dlo[3] = {0, 0, 0}, dhi[3] = {n - 1, n - 1, n - 1};

  // the register of the fine level (PeleC's getFluxReg(level + 1)), made on regrid
  pcg_fluxreg* reg = nullptr;
  int rc = pcg_fluxreg_create(nc, dlo, dhi, periodic, ratio, 1, flo, fhi, &reg);
  if (rc) return fail("pcg_fluxreg_create", rc);
  const pcg_stream_t s = nullptr;
  if ((rc = pcg_fluxreg_reset(reg, s))) return fail("pcg_fluxreg_reset", rc);  // Advance.cpp:30-31

  // the coarse level's box loop: update_flux_registers with fr_as_crse = reg
  std::vector<DevFab> cflx;
  if (!read_faces(fi, cbox, nc, cflx)) return 2;
  amrex::Array4<const amrex::Real> cf[3] = {cflx[0].array(), cflx[1].array(), cflx[2].array()};
  if ((rc = pcg_pelec::update_flux_registers(reg, nullptr, cbox, cf, dt_c, s)))
    return fail("update_flux_registers (coarse)", rc);

  // the fine level's substeps: update_flux_registers with fr_as_fine = reg
  for (int k = 0; k < nsub; ++k) {
    std::vector<DevFab> fflx;
    if (!read_faces(fi, fbox, nc, fflx)) return 2;
    amrex::Array4<const amrex::Real> ff[3] = {fflx[0].array(), fflx[1].array(), fflx[2].array()};
    if ((rc = pcg_pelec::update_flux_registers(nullptr, reg, fbox, ff, dt_f, s)))
      return fail("update_flux_registers (fine)", rc);
  }

  // post_timestep of the coarse level: reflux
  DevFab state(cbox, nc);
  if (!state.read(fi)) return 2;
  std::fclose(fi);
  if ((rc = pcg_pelec::reflux(reg, state.array(), vol, s))) return fail("reflux", rc);
  std::vector<double> out(state.n());
  if (cudaMemcpy(out.data(), state.d, out.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return 3;
  pcg_fluxreg_destroy(reg);
  std::FILE* fo = std::fopen(argv[2], "wb");
  if (!fo) return 2;
  std::fwrite(out.data(), sizeof(double), out.size(), fo);
  std::fclose(fo);
  std::printf("fluxreg_test ok: %d coarse cells, %d fine substeps\n", n * n * n, nsub);
  return 0;
}
