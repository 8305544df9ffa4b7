// pcg_types.h -- layouts shared by the host runtime and the device kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define PCG_HD __host__ __device__
#else
#define PCG_HD
#endif

namespace pcg {

// Source/IndexDefines.H:6-89 (NUM_ADV = NUM_AUX = NUM_LIN = 0)
enum { URHO = 0, UMX = 1, UMY = 2, UMZ = 3, UEDEN = 4, UEINT = 5, UTEMP = 6, UFS = 7 };
enum { QRHO = 0, QU = 1, QV = 2, QW = 3, QGAME = 4, QPRES = 5, QREINT = 6, QTEMP = 7, QFS = 8 };
enum { QGAMC = 0, QC = 1, QCSML = 2, QDPDR = 3, QDPDE = 4, QRSPEC = 5, NQAUX = 6 };
enum { GDRHO = 0, GDU = 1, GDV = 2, GDW = 3, GDPRES = 4, GDGAME = 5, NGDNV = 6 };
// Source/PeleC.H:49-57
enum { BC_INTERIOR = 0, BC_INFLOW, BC_OUTFLOW, BC_SYMMETRY, BC_SLIP_WALL, BC_NO_SLIP_WALL, BC_USER };

// Face-state layout of the traced states (qm/qp of the reference, only the components
// the path reads): rho, u, v, w, p, rho*e, Y[NS].
enum { TR_RHO = 0, TR_U = 1, TR_V = 2, TR_W = 3, TR_P = 4, TR_RE = 5, TR_Y = 6 };
// Transverse-flux layout: URHO, UMX, UMY, UMZ, UEDEN (same indices as U), then Y[NS]
// at FL_Y, then the Godunov pressure and normal velocity (qint GDPRES / GDU..GDW).
enum { FL_Y = 5 };
PCG_HD constexpr int nt_comps(int ns) { return 6 + ns; }
PCG_HD constexpr int nf_comps(int ns) { return 7 + ns; }
PCG_HD constexpr int nvar(int ns) { return 7 + ns; }
PCG_HD constexpr int qvar(int ns) { return 8 + ns; }

// Source/Constants.H:18-30
constexpr double SMALLU = 1.0e-12;
constexpr double SMALL_NUM = 1.0e-8;
constexpr double VERY_SMALL_NUM = 2.220446049250313080847263336181640625e-16 * 1e-100;

// EOS restatement constants (same as the oracle)
constexpr double RU = 8.31446261815324e7;
constexpr int NEWTON_MAXIT = 20;
constexpr double NEWTON_RTOL = 1.0e-10;
constexpr double NEWTON_TMIN = 10.0;
// Largest species count of an EOS table (the bank size of the constant-memory EOS
// tables, even so that species pairs fill it). The build sets it from the largest
// species count it compiles kernels for; every unit and the host see the same value.
#ifndef PCG_MAXNS
#define PCG_MAXNS 16
#endif
constexpr int MAXNS = PCG_MAXNS;
static_assert(MAXNS % 2 == 0, "PCG_MAXNS must be even");
// The kernels address a view with 32-bit element offsets: every view the host passes them
// (workspace arrays and the caller's arrays) spans fewer elements than this.
constexpr int64_t kMaxViewElems = 2147483647;

struct EosConst {
  int kind;  // 0 gamma law, 1 NASA-7 mixture
  int nspec;
  int uniform_tmid;  // 1: every species switches NASA-7 range at tmid[0]
  double gamma;
  double imw[MAXNS];
  double tmid[MAXNS];
  double cvc[MAXNS][2][5];
  double ec[MAXNS][2][6];
  float gammaf;
  float imwf[MAXNS];
  float tmidf[MAXNS];
  float cvcf[MAXNS][2][5];
  float ecf[MAXNS][2][6];
  // the same FP32 coefficients species-minor (zero past nspec), so that species 2m and
  // 2m+1 form one aligned pair for the packed FP32 arithmetic (FFMA2)
  alignas(8) float cvp[2][5][MAXNS];
  alignas(8) float ecp[2][6][MAXNS];
  alignas(8) float imwp[MAXNS];
};

// A strided block of memory addressed like amrex::Array4 (element type decided by the
// kernel that reads it): p[(i-b0) + (j-b1)*js + (k-b2)*ks + n*ns].
// Blocked workspace arrays (the traced states and the face fluxes the flux stages pass
// on) use the same linear cell index L = (i-b0) + (j-b1)*js + (k-b2)*ks but group the
// cells in blocks of kCellBlock consecutive L, each block holding all its components one
// after the other: element (L, n) at p[(L / 32) * ns + n * 32 + L % 32], ns = 32 * ncomp.
// A warp reading one component of 32 consecutive cells still reads 128 contiguous bytes,
// and the components of a cell are compile-time offsets from its first one.
constexpr int kCellBlock = 32;
struct View {
  void* p;
  int64_t js, ks, ns;
  int32_t b[3];
  int32_t blocked;  // 1: blocked layout (ns is the block stride)
};

// Everything one box of a launch needs. Workspace views point into the library's
// workspace; in/out views may be the caller's arrays.
struct Region {
  int32_t lo[3], hi[3];
  int32_t domlo[3], domhi[3], bclo[3], bchi[3];
  double dx[3];
  double dt;        // used unless StageArgs::dt_dev or dt_ptr is set
  const double* dt_ptr;  // device pointer to this region's own timestep (batched steps)
  double area_u[3]; // uniform face areas (used when area[d].p == nullptr)
  double vol_u;     // uniform volume (used when vol.p == nullptr)
  View uin;         // conserved state, double, >= 4 ghosts
  View uout;        // hydro source, double, valid box
  View q;           // primitive state, double, QVAR comps on >= grow(box,4)
  View qa;          // auxiliary state, double, NQAUX comps
  View srcq;        // primitive sources (p == nullptr: none)
  View prep;        // flattening and trace sound speed on grow(box,1), compute type
  View qf;          // mixed form: FP32 copy of q on grow(box,3) in trace-state layout
                    // (rho, u, v, w, p - p0, rho e, Y), p == nullptr otherwise
  View divu;        // nodal div u on the box's nodes, double
  View area[3];     // face areas (p == nullptr: uniform)
  View vol;         // cell volumes (p == nullptr: uniform)
  View trm[3];      // traced minus (left) states on the d-faces, compute type
  View trp[3];      // traced plus (right) states on the d-faces, compute type
  View fi[3];       // initial d-fluxes, compute type
  View fdo[3][3];   // d-fluxes from d-states corrected by o-fluxes, compute type
  View ff[3];       // final fluxes, double, NVAR comps (area-weighted)
  View qec[3];      // Godunov pressure and normal velocity at final faces, double
  int32_t zero_uout; // 1: write uout (=), 0: accumulate (+=)
  int32_t qf_in_prep; // 1: k_prep writes qf (no ctoprim stage), 0: k_ctoprim writes it
  int32_t ff_single;  // 1: ff/qec are FP32 with the pressure as deviation from p0
  int32_t qf_grow;    // qf covers grow(box, qf_grow): 3, or 4 for the 7-point WENO trace
  // pc_umeth_3D on its own (pcg_umeth): the final stage writes the unadjusted Godunov
  // fluxes into ff (FP64, caller's arrays, UTEMP untouched) and the face states into qec
  // (the caller's NGDNV-component arrays, GDRHO untouched), and p div u goes to pdivu
  // instead of the flux divergence
  int32_t umeth;
  int32_t pad2;
  View pdivu;       // umeth: p div u on the box, double
  View src;         // pcg_srctoprim: conserved sources, double, NVAR comps
};

// A run of thread blocks of one stage working on one region (and one variant, e.g.
// a direction or a (direction, other direction) pair) over the index box
// [lo, lo + n).
// Blocks (of 128 threads) of the stages that share a cell's transverse correction
// between its two faces (k_flux1, k_flux2): x-faces one face per thread; y- and
// z-faces one thread per FACE_MARCH consecutive faces along their direction.
constexpr int FACE_MARCH = 4;
PCG_HD constexpr int64_t face_threads(int d, const int32_t n[3]) {
  return d == 0 ? int64_t(n[0]) * n[1] * n[2]
                : int64_t(n[0]) * n[d == 1 ? 2 : 1] * ((n[d] + FACE_MARCH - 1) / FACE_MARCH);
}
PCG_HD constexpr int64_t face_tiles(int d, const int32_t n[3]) { return (face_threads(d, n) + 127) / 128; }
// k_flux1 shares corrections in the FP32 form only (element size of the compute type);
// the FP64 forms run one face per thread.
PCG_HD constexpr bool flux1_shared(size_t esz) { return esz == 4; }

struct Seg {
  int32_t region;
  int32_t variant;
  int32_t lo[3];
  int32_t n[3];
  int64_t count;
  int64_t blk0;  // first block of this segment within the launch
};

struct StageArgs {
  const Region* regions;
  const Seg* segs;
  int32_t nseg;
  int32_t ppm_type;
  int32_t plm_iorder;
  int32_t use_flattening;
  int32_t use_hybrid_weno;
  int32_t weno_scheme;
  int32_t umeth;  // the call is pcg_umeth (see Region::umeth)
  double difmag;
  const double* dt_dev;  // nullptr: each region's dt
  double* partial;       // fused step tail: one timestep minimum per block
  const void* tmaps;     // TMA-staged trace: 3 tensor maps (x, y, z boxes) per region
  int32_t* err;          // device error word: bit 0 set when a bounded TMA wait gave up
};
// The tiles of the TMA-staged trace, one per block of 128 threads: 32 cells along x by 4
// along y (x and y traces) or along z (z trace), so that the 4 warps of a block are the
// tile's 4 rows and the traced direction's neighbours are lanes (x) or warps (y, z). The
// staged box adds the +-2 cells of the stencil along the traced direction, and along x up
// to 3 more cells, because a box starts at a 16-byte boundary of the array.
constexpr int kTraceTileX = 32;
PCG_HD constexpr int trace_tile_y(int d) { return d == 2 ? 1 : 4; }
PCG_HD constexpr int trace_tile_z(int d) { return d == 2 ? 4 : 1; }
PCG_HD constexpr int trace_box_x(int d) { return d == 0 ? 40 : 36; }
PCG_HD constexpr int trace_box_y(int d) { return d == 0 ? 4 : d == 1 ? 8 : 1; }
PCG_HD constexpr int trace_box_z(int d) { return d == 2 ? 8 : 1; }
PCG_HD constexpr int trace_box_cells(int d) { return trace_box_x(d) * trace_box_y(d) * trace_box_z(d); }
// The tiled trace's shared arrays (the staged primitives, slopes and interface values of
// a tile) grow with the species count: about 37 KB at 9 species, past 12 species more
// than the 48 KB of static shared memory of a block. Larger counts trace per cell.
PCG_HD constexpr bool trace_tile_species(int ns) { return ns <= 12; }
// Bytes of one CUtensorMap (the layout of the driver's opaque type).
constexpr int kTensorMapBytes = 128;

// One box for the auxiliary kernels (timestep, state update).
struct AuxBox {
  int32_t lo[3], hi[3];
  double dx[3];
  double dt;
  View uin;   // S_old
  View uout;  // hydro source
  View snew;  // S_new (may alias uin)
};

// One box of a batched ghost fill: the ghost cells of grow(domain box, ng) of its state.
struct FillBox {
  View state;
  int32_t dlo[3], dhi[3];
  int32_t periodic;  // bit d set: periodic wrap in direction d, else zero-gradient
  int32_t pad;
  int64_t count;     // ghost cells
  int64_t blk0;      // first block of this box within the launch
};

struct AuxArgs {
  const AuxBox* boxes;
  const Seg* segs;
  int32_t nseg;
  double* partial;      // timestep: one minimum per block
  int64_t npartial;
  double cfl;
  double* dt_out;       // timestep result (device)
  const double* dt_in;  // state update: device dt (nullptr: per-box dt)
  View state;           // ghost fill: domain FAB
  int32_t dlo[3], dhi[3], ng, ncomp;
  int32_t periodic;     // ghost fill: bit d set when direction d is periodic
  const FillBox* fills; // batched ghost fill
  int32_t nfill;
  int32_t pad;
  View dst;               // device box copy: destination (state is the source)
  const pcg::Seg* bsegs;  // per-box timestep: the advance segments of each region
  double* dt_boxes;       // per-box timestep result (device, one per region)
};

}  // namespace pcg
