// pcg_host.cu -- host runtime behind include/pcg_hydro.h: argument checks, EOS
// tables, workspace layout, launch plans and the C entry points.
//
// A launch plan lays out, for every box (region) of a call, the intermediate arrays
// of the advance in one device workspace and builds per-stage segment tables (see
// pcg_types.h). One-shot calls allocate the workspace stream-ordered on the caller's
// stream from a memory pool the library owns per device, which keeps its memory
// between calls (the role amrex::The_Async_Arena plays in the reference);
// pcg_plan objects keep theirs for repeated steps so that a step can be captured in a
// CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <deque>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "../../include/pcg_hydro.h"
#include "pcg_types.h"

#include "pcg_units.h"

// The kernel translation units, one per (arithmetic, species count), register their
// entry points here at library load (pcg_dispatch.cuh); the table is written only by
// those static initialisers and read afterwards.
namespace pcg {
namespace {
struct UnitTable {
  std::vector<UnitEntry> units;
};
UnitTable& unit_table() {
  static UnitTable t;
  return t;
}
}  // namespace
void register_unit(const UnitEntry& u) { unit_table().units.push_back(u); }
}  // namespace pcg

namespace {
const pcg::UnitEntry* find_unit(int kind, int ns) {
  for (const pcg::UnitEntry& u : pcg::unit_table().units)
    if (u.kind == kind && u.ns == ns) return &u;
  return nullptr;
}
// true when the build holds the kernels of every form for this species count
bool species_built(int ns) {
  return find_unit(pcg::UNIT_STRICT, ns) && find_unit(pcg::UNIT_FAST, ns) && find_unit(pcg::UNIT_MIXED, ns);
}
// the species counts with kernels, ascending, as text ("1, 9")
std::string species_list() {
  std::vector<int> v;
  for (const pcg::UnitEntry& u : pcg::unit_table().units)
    if (u.kind == pcg::UNIT_STRICT && species_built(u.ns)) v.push_back(u.ns);
  std::sort(v.begin(), v.end());
  std::string out;
  for (size_t k = 0; k < v.size(); ++k) out += (k ? ", " : "") + std::to_string(v[k]);
  return out;
}
}  // namespace

// Routing by species count: pcg_strict = FP64 reference order (and the FP64 auxiliary
// kernels), pcg_fast = FMA-contracted FP64 stages (single == false) or the mixed form's
// FP32 stages (single == true), and the FP64 step tail of both fast forms. A species
// count without kernels is cudaErrorInvalidValue (the entry points refuse it earlier
// with PCG_EUNSUPPORTED).
namespace pcg_strict {
// slot 0 holds the gamma law (species count 1), slot 1 the mixture table of e.nspec
// species: each goes to the units of that species count
cudaError_t upload_eos(int slot, const pcg::EosConst& e) {
  const pcg::UnitEntry* u = find_unit(pcg::UNIT_STRICT, slot == 0 ? 1 : e.nspec);
  return u ? u->upload_eos(slot, e) : cudaErrorInvalidValue;
}
cudaError_t launch_stage(int stage, int ns, bool single, const pcg::StageArgs& a, int64_t nblocks, int variant,
                         cudaStream_t s) {
  const pcg::UnitEntry* u = find_unit(pcg::UNIT_STRICT, ns);
  return u ? u->launch_stage(stage, ns, single, a, nblocks, variant, s) : cudaErrorInvalidValue;
}
cudaError_t launch_advance(int ns, const pcg::StageArgs& a, int64_t nblocks, int variant, cudaStream_t s) {
  const pcg::UnitEntry* u = find_unit(pcg::UNIT_STRICT, ns);
  return u ? u->launch_advance(ns, a, nblocks, variant, s) : cudaErrorInvalidValue;
}
cudaError_t launch_aux(int which, int ns, const pcg::AuxArgs& a, int64_t nblocks, cudaStream_t s) {
  const pcg::UnitEntry* u = find_unit(pcg::UNIT_STRICT, ns);
  return u ? u->launch_aux(which, ns, a, nblocks, s) : cudaErrorInvalidValue;
}
}  // namespace pcg_strict
namespace pcg_fast {
cudaError_t upload_eos(int slot, const pcg::EosConst& e) {
  const int ns = slot == 0 ? 1 : e.nspec;
  const pcg::UnitEntry* f = find_unit(pcg::UNIT_FAST, ns);
  const pcg::UnitEntry* m = find_unit(pcg::UNIT_MIXED, ns);
  if (!f || !m) return cudaErrorInvalidValue;
  cudaError_t r = f->upload_eos(slot, e);
  return r != cudaSuccess ? r : m->upload_eos(slot, e);
}
cudaError_t launch_stage(int stage, int ns, bool single, const pcg::StageArgs& a, int64_t nblocks, int variant,
                         cudaStream_t s) {
  const pcg::UnitEntry* u = find_unit(single ? pcg::UNIT_MIXED : pcg::UNIT_FAST, ns);
  return u ? u->launch_stage(stage, ns, single, a, nblocks, variant, s) : cudaErrorInvalidValue;
}
cudaError_t launch_advance(int ns, const pcg::StageArgs& a, int64_t nblocks, int variant, cudaStream_t s) {
  const pcg::UnitEntry* u = find_unit(pcg::UNIT_FAST, ns);
  return u ? u->launch_advance(ns, a, nblocks, variant, s) : cudaErrorInvalidValue;
}
}  // namespace pcg_fast

namespace {

enum { K_CTOPRIM = 0, K_PREP, K_TRACE, K_FLUX0, K_FLUX1, K_FLUX2, K_CONSUP, K_NSTAGE };
// launches that are not stages of their own: the low-order inflow/user_bc faces, run as
// part of stage K_FLUX2 right after it, pc_srctoprim (pcg_srctoprim), and the TMA-staged
// trace that stands in for stage K_TRACE in the mixed form
enum { K_LOWBC = K_NSTAGE, K_SRCQ, K_TRACE_TILE, K_NKIND };
enum { AUX_ESTDT = 0, AUX_ESTDT_FINAL, AUX_UPDATE, AUX_FILL, AUX_FILL_BOXES, AUX_ESTDT_BOXES, AUX_COPY };
constexpr int kThreads = 128;
constexpr size_t kAlign = 256;

thread_local std::string g_err;

// Launch-variant table: [precision_mode][species slot][stage] -> variant index of
// kMinBlocks (pcg_kernels.cuh). Defaults measured on B200 for the production flame
// level; pcg_set_launch_variant (the autotuner) overrides them. The mixed form's trace
// has three more variants: 3-5 run the TMA-staged tiled trace (K_TRACE_TILE) with the
// register budgets 0-2.
constexpr int kTileVariant = 3;
std::mutex g_var_mu;
int g_variant[3][2][7] = {
  {{0, 0, 2, 0, 1, 2, 1}, {2, 0, 1, 1, 1, 0, 2}},  // FP64 reference order
  {{1, 0, 1, 0, 0, 0, 1}, {1, 0, 1, 0, 0, 0, 1}},  // FP64 with FMA
  {{0, 0, 2, 0, 1, 0, 1}, {2, 0, 2, 2, 2, 1, 2}},  // mixed
};
int max_variant(int prec, int stage) { return (prec == PCG_PREC_MIXED && stage == K_TRACE) ? 5 : 2; }
int variant_of(int prec, int ns, int stage) {
  std::lock_guard<std::mutex> lk(g_var_mu);
  return g_variant[prec][ns == 1 ? 0 : 1][stage];
}

// Stream-ordered workspace pool per device. Its release threshold is unbounded, so
// memory freed by one call is reused by the next without returning to the driver (the
// default pool would trim it at every synchronisation); pcg_trim_workspace hands it back.
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};

cudaError_t workspace_pool(cudaMemPool_t* pool) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if ((e = cudaMemPoolCreate(&p, &props)) != cudaSuccess) return e;
    uint64_t thr = UINT64_MAX;
    if ((e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &thr)) != cudaSuccess) {
      cudaMemPoolDestroy(p);
      return e;
    }
    g_pool[dev] = p;
  }
  *pool = g_pool[dev];
  return cudaSuccess;
}

// Allocation sizes are rounded up to size classes (from 1 MiB on, 4 to 7 units of a power
// of two, at most 25 % over): the one-shot calls of a serving loop ask for a different
// workspace size nearly every time, and without classes the pool keeps mapping new
// memory for sizes that no freed block fits (tens of milliseconds per call, measured),
// while a freed block of a class serves every later request of that class.
size_t size_class(size_t bytes) {
  if (bytes <= (size_t(1) << 20)) return bytes;
  int k = 63 - __builtin_clzll(bytes);  // 2^k <= bytes < 2^(k+1)
  const size_t unit = size_t(1) << (k - 2);
  return (bytes + unit - 1) / unit * unit;
}

cudaError_t ws_alloc(void** p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool = nullptr;
  cudaError_t e = workspace_pool(&pool);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(p, size_class(bytes), pool, s);
}

// Pinned staging buffers for the table uploads of one-shot calls. A copy from pageable
// host memory goes through the driver's few staging buffers, so once a handful of calls
// are queued on a busy stream the next one blocks until the device has drained the
// earlier copies: the host then waits for the device call after call. Here each upload
// takes a pinned buffer that no queued copy still reads (an event recorded after its
// last copy has completed), or a new one; buffers are kept for the life of the process.
struct Staging {
  void* host = nullptr;
  size_t bytes = 0;
  int device = -1;
  cudaEvent_t done = nullptr;
};
std::mutex g_stage_mu;
std::deque<Staging> g_stage;

cudaError_t upload(void* dst, const void* src, size_t n, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cs);
  if (e != cudaSuccess) return e;
  // under stream capture: a plain copy (the reuse of a staging buffer is tracked with an
  // event recorded at run time, which a captured graph does not provide)
  if (cs != cudaStreamCaptureStatusNone) return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, s);
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_stage_mu);
  Staging* pick = nullptr;
  for (Staging& b : g_stage) {
    if (b.device != dev || b.bytes < n) continue;
    const cudaError_t q = cudaEventQuery(b.done);
    if (q == cudaErrorNotReady) {
      if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();
      continue;
    }
    if (q != cudaSuccess) return q;
    pick = &b;
    break;
  }
  if (!pick) {
    Staging b;
    b.device = dev;
    b.bytes = std::max<size_t>((n + 65535) / 65536 * 65536, 65536);
    if ((e = cudaHostAlloc(&b.host, b.bytes, cudaHostAllocPortable)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming)) != cudaSuccess) {
      cudaFreeHost(b.host);
      return e;
    }
    g_stage.push_back(b);
    pick = &g_stage.back();
  }
  std::memcpy(pick->host, src, n);
  if ((e = cudaMemcpyAsync(dst, pick->host, n, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  return cudaEventRecord(pick->done, s);
}

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CUDA_TRY(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      cudaGetLastError();                                                               \
      return fail(e_ == cudaErrorMemoryAllocation ? PCG_ENOMEM : PCG_ECUDA, "%s: %s", #call, \
                  cudaGetErrorString(e_));                                              \
    }                                                                                   \
  } while (0)

// ------------------------------------------------------------------ EOS tables
struct EosState {
  std::mutex mu;
  bool set[2] = {false, false};
  pcg::EosConst c[2];
  uint64_t version[2] = {0, 0};
  uint64_t uploaded[64][2] = {};  // per device
};
EosState& eos_state() {
  static EosState s;
  return s;
}

int eos_slot(int nspec) { return nspec == 1 ? 0 : 1; }

int ensure_eos(int nspec) {
  EosState& es = eos_state();
  const int slot = eos_slot(nspec);
  std::lock_guard<std::mutex> lk(es.mu);
  if (!es.set[slot] || es.c[slot].nspec != nspec)
    return fail(PCG_ENOEOS, "no EOS table set for nspec=%d (pcg_set_eos_gamma / pcg_set_eos_nasa7)", nspec);
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(PCG_EINVAL, "device index %d out of range", dev);
  if (es.uploaded[dev][slot] != es.version[slot]) {
    CUDA_TRY(pcg_strict::upload_eos(slot, es.c[slot]));
    CUDA_TRY(pcg_fast::upload_eos(slot, es.c[slot]));
    es.uploaded[dev][slot] = es.version[slot];
  }
  return PCG_OK;
}

int store_eos(int slot, const pcg::EosConst& c) {
  EosState& es = eos_state();
  {
    std::lock_guard<std::mutex> lk(es.mu);
    es.c[slot] = c;
    es.set[slot] = true;
    es.version[slot] += 1;
  }
  return ensure_eos(c.nspec);
}

// ------------------------------------------------------------------ boxes & views
struct IBox {
  int lo[3], hi[3];
  int64_t n(int d) const { return hi[d] - lo[d] + 1; }
  int64_t cells() const { return n(0) * n(1) * n(2); }
  bool ok() const { return hi[0] >= lo[0] && hi[1] >= lo[1] && hi[2] >= lo[2]; }
};
IBox mkbox(const int32_t* lo, const int32_t* hi) {
  IBox b;
  for (int d = 0; d < 3; ++d) { b.lo[d] = lo[d]; b.hi[d] = hi[d]; }
  return b;
}
IBox grow(IBox b, int n) {
  for (int d = 0; d < 3; ++d) { b.lo[d] -= n; b.hi[d] += n; }
  return b;
}
IBox grow_dir(IBox b, int d, int n) { b.lo[d] -= n; b.hi[d] += n; return b; }
IBox nodes(IBox b, int d) { b.hi[d] += 1; return b; }

pcg::View view_of(const pcg_array4* a) {
  pcg::View v{};
  if (!a || !a->p) return v;
  v.p = a->p;
  v.js = a->jstride;
  v.ks = a->kstride;
  v.ns = a->nstride;
  for (int d = 0; d < 3; ++d) v.b[d] = a->begin[d];
  return v;
}

bool covers(const pcg_array4* a, const IBox& b, int ncomp) {
  if (!a || !a->p) return false;
  for (int d = 0; d < 3; ++d)
    if (a->begin[d] > b.lo[d] || a->end[d] <= b.hi[d]) return false;
  return a->ncomp >= ncomp;
}

// Largest element offset of an array from its begin corner (the kernels' 32-bit offsets).
int64_t max_offset(const pcg_array4* a) {
  return int64_t(a->end[0] - a->begin[0] - 1) + int64_t(a->end[1] - a->begin[1] - 1) * a->jstride +
         int64_t(a->end[2] - a->begin[2] - 1) * a->kstride + int64_t(a->ncomp - 1) * a->nstride;
}

int check_array(const char* what, const pcg_array4* a, const IBox& b, int ncomp) {
  if (a && a->p && (max_offset(a) > pcg::kMaxViewElems || a->jstride > pcg::kMaxViewElems ||
                    a->kstride > pcg::kMaxViewElems || a->nstride > pcg::kMaxViewElems))
    return fail(PCG_EINVAL, "%s spans more than 2^31 elements (the kernels address arrays with 32-bit offsets)",
                what);
  if (!covers(a, b, ncomp))
    return fail(PCG_EINVAL, "%s must cover [%d,%d,%d]-[%d,%d,%d] with %d components", what, b.lo[0], b.lo[1],
                b.lo[2], b.hi[0], b.hi[1], b.hi[2], ncomp);
  return PCG_OK;
}

int check_params(const pcg_hydro_params* p) {
  if (!p) return fail(PCG_EINVAL, "params is NULL");
  if (!species_built(p->nspec))
    return fail(PCG_EUNSUPPORTED, "nspec=%d: this build has kernels for %s species", p->nspec, species_list().c_str());
  if (p->ppm_type != 0 && p->ppm_type != 1) return fail(PCG_EINVAL, "PeleC::ppm_type must be 0 (PLM) or 1 (PPM)");
  if (p->use_hybrid_weno && p->ppm_type != 1)
    return fail(PCG_EINVAL, "PeleC::ppm_type must be 1 (PPM) to use WENO method");
  if (p->use_hybrid_weno && (p->weno_scheme < 0 || p->weno_scheme > 3))
    return fail(PCG_EINVAL, "weno_scheme %d: 0 WENO-JS5, 1 WENO-Z5, 2 WENO-Z7 or 3 WENO-Z3", p->weno_scheme);
  if (p->ppm_type == 0 && p->plm_iorder != 1 && p->plm_iorder != 2 && p->plm_iorder != 4)
    return fail(PCG_EINVAL, "plm_iorder must be 1, 2 or 4");
  if (p->precision_mode < PCG_PREC_FP64 || p->precision_mode > PCG_PREC_MIXED)
    return fail(PCG_EINVAL, "precision_mode %d", p->precision_mode);
  return PCG_OK;
}

int check_box_common(const IBox& bx, const double* dx, double dt, const int32_t* bclo, const int32_t* bchi) {
  if (!bx.ok()) return fail(PCG_EINVAL, "empty box");
  for (int d = 0; d < 3; ++d) {
    if (!(dx[d] > 0.0) || !std::isfinite(dx[d])) return fail(PCG_EINVAL, "dx[%d] must be positive", d);
    if (bclo[d] < PCG_BC_INTERIOR || bclo[d] > PCG_BC_USER || bchi[d] < PCG_BC_INTERIOR || bchi[d] > PCG_BC_USER)
      return fail(PCG_EINVAL, "unknown boundary type in direction %d", d);
  }
  if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(PCG_EINVAL, "dt must be finite and >= 0");
  return PCG_OK;
}

// ------------------------------------------------------------------ launch plans
struct BoxIn {
  IBox bx;
  int domlo[3], domhi[3], bclo[3], bchi[3];
  double dx[3];
  double dt;
  pcg::View uin, uout, q, qa, srcq, area[3], vol, flx[3];
  pcg::View qec[3], pdivu;  // pcg_umeth: the caller's face states and p div u
  bool internal_q;  // ctoprim into the workspace
  bool zero_uout;
  bool umeth = false;  // pc_umeth_3D alone: raw fluxes, qec and pdivu (see pcg::Region::umeth)
};

struct Layout {
  bool oversize = false;  // a workspace array would span 2^31 elements or more
  bool tile_trace = false;  // the mixed form's trace runs as TMA-staged tiles (K_TRACE_TILE)
  int ns = 1;
  int umeth = 0;  // the plan is a pcg_umeth call
  size_t esz = 8;  // compute-type size of the intermediates
  size_t ws_bytes = 0;
  std::vector<pcg::Region> regions;
  std::vector<pcg::Seg> segs[K_NKIND];
  int64_t nblocks[K_NKIND] = {};
};

// A workspace array of nc components over box b: Array4 layout, or with blocked != 0 the
// blocked layout of pcg::View (cells in blocks of pcg::kCellBlock, all components of a
// block together), which the arrays the flux stages pass on use.
// With pad_rows the rows of an Array4-layout array are padded to a multiple of 4 elements
// (16 bytes for FP32), as the TMA tensor maps of the staged trace need.
size_t take(Layout& L, const IBox& b, int nc, size_t esz, pcg::View& v, bool blocked = false, bool pad_rows = false) {
  const size_t off = (L.ws_bytes + kAlign - 1) / kAlign * kAlign;
  v.p = reinterpret_cast<void*>(off);  // rebased once the workspace exists
  v.js = pad_rows ? (b.n(0) + 3) / 4 * 4 : b.n(0);
  v.ks = v.js * b.n(1);
  const int64_t cells = blocked ? (b.cells() + pcg::kCellBlock - 1) / pcg::kCellBlock * pcg::kCellBlock
                                : v.ks * b.n(2);
  v.ns = blocked ? int64_t(pcg::kCellBlock) * nc : cells;
  v.blocked = blocked ? 1 : 0;
  for (int d = 0; d < 3; ++d) v.b[d] = b.lo[d];
  L.ws_bytes = off + size_t(cells) * nc * esz;
  if (cells * nc > pcg::kMaxViewElems) L.oversize = true;
  return off;
}

void add_seg(Layout& L, int stage, int region, int variant, const IBox& b) {
  pcg::Seg s{};
  s.region = region;
  s.variant = variant;
  for (int d = 0; d < 3; ++d) { s.lo[d] = b.lo[d]; s.n[d] = (int)b.n(d); }
  s.count = b.cells();
  s.blk0 = L.nblocks[stage];
  L.segs[stage].push_back(s);
  const bool tiled = stage == K_FLUX2 || (stage == K_FLUX1 && pcg::flux1_shared(L.esz));
  L.nblocks[stage] += tiled ? pcg::face_tiles(variant, s.n) : (s.count + kThreads - 1) / kThreads;
}

// Work order within a launch. Blocks start roughly in launch order, so the order of the
// segments decides which data is live in L2 at the same time.
// (1) The final fluxes of all three directions read the state and the nodal div u
// (artificial viscosity). In a region whose state would not stay in L2 between its
// direction segments (kOrderRegionBytes) the k_flux2 direction segments are therefore
// interleaved in slabs of kOrderSlab z-planes (x, y, z of one slab, then the next slab)
// so that a slab's state comes from DRAM once. Measured on the 128^3 flame level (mixed
// form): flux2 0.672 -> 0.657 ms. The same interleave slowed the stages whose
// directions run different code (flux1 0.661 -> 0.726 ms, trace 0.631 -> 0.658, flux0
// 0.228 -> 0.245), so they keep one segment per direction (PCG_ORDER_SLABS: bit K_* of
// the stages that interleave).
// (2) Successive stages alternate their traversal direction (prep, flux0 and flux2 run
// their segments in reverse order, PCG_ORDER_REVERSE), so that the data a stage wrote
// last, still in L2, is what the next stage reads first (step 2.960 -> 2.953 ms alone,
// 2.935 ms with (1)).
// Every face and cell is computed by the same expressions whatever the order, so the
// results do not depend on it.
constexpr int kOrderSlab = 8;
constexpr int64_t kOrderRegionBytes = int64_t(64) << 20;
#ifndef PCG_ORDER_SLABS
#define PCG_ORDER_SLABS 0x20
#endif
#ifndef PCG_ORDER_REVERSE
#define PCG_ORDER_REVERSE 0x2A
#endif
constexpr unsigned kOrderSlabStages = PCG_ORDER_SLABS, kOrderReverseStages = PCG_ORDER_REVERSE;

// The segments of one stage over the direction boxes b[0..2] of region `region`
// (variant = direction), slab-interleaved when `slabs` is set.
void add_dir_segs(Layout& L, int stage, int region, const IBox b[3], bool slabs, int z0) {
  if (!slabs || !((kOrderSlabStages >> stage) & 1u)) {
    for (int d = 0; d < 3; ++d) add_seg(L, stage, region, d, b[d]);
    return;
  }
  int zlo = b[0].lo[2], zhi = b[0].hi[2];
  for (int d = 1; d < 3; ++d) {
    zlo = std::min(zlo, b[d].lo[2]);
    zhi = std::max(zhi, b[d].hi[2]);
  }
  // slabs of kOrderSlab planes on the grid z0 + m kOrderSlab (z0: the region's first
  // valid plane), so that march chunks of the z-faces start on the region's 4-face grid
  int zs = z0;
  while (zs > zlo) zs -= kOrderSlab;
  for (; zs <= zhi; zs += kOrderSlab) {
    for (int d = 0; d < 3; ++d) {
      IBox c = b[d];
      c.lo[2] = std::max(c.lo[2], zs);
      c.hi[2] = std::min(c.hi[2], zs + kOrderSlab - 1);
      if (c.ok()) add_seg(L, stage, region, d, c);
    }
  }
}

// The segments of a one-variant stage over box b: one, or z-slabs of kOrderSlab planes
// on the same grid as add_dir_segs.
void add_slab_segs(Layout& L, int stage, int region, const IBox& b, bool slabs, int z0) {
  if (!slabs || !((kOrderSlabStages >> stage) & 1u)) {
    add_seg(L, stage, region, 0, b);
    return;
  }
  int zs = z0;
  while (zs > b.lo[2]) zs -= kOrderSlab;
  for (; zs <= b.hi[2]; zs += kOrderSlab) {
    IBox c = b;
    c.lo[2] = std::max(c.lo[2], zs);
    c.hi[2] = std::min(c.hi[2], zs + kOrderSlab - 1);
    if (c.ok()) add_seg(L, stage, region, 0, c);
  }
}

// Reverse the launch order of a stage's segments (block offsets renumbered).
void reverse_segs(Layout& L, int stage) {
  std::vector<pcg::Seg>& v = L.segs[stage];
  const size_t n = v.size();
  std::vector<int64_t> nb(n);
  for (size_t i = 0; i < n; ++i) nb[i] = (i + 1 < n ? v[i + 1].blk0 : L.nblocks[stage]) - v[i].blk0;
  std::reverse(v.begin(), v.end());
  std::reverse(nb.begin(), nb.end());
  int64_t b = 0;
  for (size_t i = 0; i < n; ++i) {
    v[i].blk0 = b;
    b += nb[i];
  }
}

// The tiled trace of direction d over g1 = grow(box,1), as K_TRACE_TILE segments: the up
// to three disjoint strips that full tiles cannot cover, along x, y and z (variant d:
// one cell per thread, read from global memory), and the full tiles of the rest
// (variant 3 + d).
void add_trace_tiles(Layout& L, int region, int d, const IBox& g1) {
  const int tn[3] = {pcg::kTraceTileX, pcg::trace_tile_y(d), pcg::trace_tile_z(d)};
  int64_t core[3];
  for (int e = 0; e < 3; ++e) core[e] = g1.n(e) / tn[e] * tn[e];
  const bool tiles = core[0] > 0 && core[1] > 0 && core[2] > 0;
  if (!tiles) core[0] = 0;  // no tile: the x strip is all of g1
  // strip e: cells past the core along e, inside the core along the directions before e
  for (int e = 0; e < 3; ++e) {
    IBox b = g1;
    b.lo[e] = g1.lo[e] + (int)core[e];
    for (int f = 0; f < e; ++f) b.hi[f] = g1.lo[f] + (int)core[f] - 1;
    bool empty = false;
    for (int f = 0; f < 3; ++f) empty = empty || b.n(f) <= 0;
    if (!empty) add_seg(L, K_TRACE_TILE, region, d, b);
    if (!tiles) break;
  }
  if (!tiles) return;
  pcg::Seg sg{};
  sg.region = region;
  sg.variant = 3 + d;
  for (int e = 0; e < 3; ++e) {
    sg.lo[e] = g1.lo[e];
    sg.n[e] = (int)(core[e] / tn[e]);
  }
  sg.count = int64_t(sg.n[0]) * sg.n[1] * sg.n[2];
  sg.blk0 = L.nblocks[K_TRACE_TILE];
  L.segs[K_TRACE_TILE].push_back(sg);
  L.nblocks[K_TRACE_TILE] += sg.count;
}

void build_layout(Layout& L, const std::vector<BoxIn>& boxes, const pcg_hydro_params* prm) {
  const int ns = prm->nspec;
  const bool single = prm->precision_mode == PCG_PREC_MIXED;
  // the 7-point WENO trace of a cell of grow(box,1) reads primitives on grow(box,4)
  const int qf_grow = (prm->use_hybrid_weno && prm->ppm_type == 1 && prm->weno_scheme == 2) ? 4 : 3;
  L.ns = ns;
  L.esz = single ? 4 : 8;
  // the mixed form traces from TMA-staged shared-memory tiles of its FP32 primitive copy
  // (PPM without hybrid WENO, and PLM)
  L.tile_trace = single && !prm->use_hybrid_weno && pcg::trace_tile_species(ns);
  const int nt = pcg::nt_comps(ns), nf = pcg::nf_comps(ns), nv = pcg::nvar(ns), nq = pcg::qvar(ns);
  for (size_t r = 0; r < boxes.size(); ++r) {
    const BoxIn& B = boxes[r];
    pcg::Region R{};
    for (int d = 0; d < 3; ++d) {
      R.lo[d] = B.bx.lo[d];
      R.hi[d] = B.bx.hi[d];
      R.domlo[d] = B.domlo[d];
      R.domhi[d] = B.domhi[d];
      R.bclo[d] = B.bclo[d];
      R.bchi[d] = B.bchi[d];
      R.dx[d] = B.dx[d];
    }
    R.dt = B.dt;
    R.area_u[0] = B.dx[1] * B.dx[2];
    R.area_u[1] = B.dx[0] * B.dx[2];
    R.area_u[2] = B.dx[0] * B.dx[1];
    R.vol_u = B.dx[0] * B.dx[1] * B.dx[2];
    R.uin = B.uin;
    R.uout = B.uout;
    R.srcq = B.srcq;
    R.vol = B.vol;
    for (int d = 0; d < 3; ++d) R.area[d] = B.area[d];
    R.zero_uout = B.zero_uout ? 1 : 0;
    const IBox g4 = grow(B.bx, 4), g1 = grow(B.bx, 1);
    // direction segments interleaved in z-slabs for large regions (see add_dir_segs)
    const bool slabs = g1.cells() * nv * 8 > kOrderRegionBytes && B.bx.n(2) >= 2 * kOrderSlab;
    const int z0 = B.bx.lo[2];
    IBox sb[3];
    if (B.internal_q) {
      // the mixed form keeps no FP64 primitive array: its stages read the FP32 copy
      if (!single) take(L, g4, nq, 8, R.q);
      take(L, g4, pcg::NQAUX, 8, R.qa);
      add_seg(L, K_CTOPRIM, (int)r, 0, g4);
    } else {
      R.q = B.q;
      R.qa = B.qa;
    }
    take(L, g1, 2, L.esz, R.prep);
    if (single) {
      // mixed form: the FP32 primitive copy the trace reads, written by k_ctoprim, or by
      // k_prep when the caller supplies q (pcg_umdrv)
      // prep's flattening reads +-3 cells around grow(box,1) from this copy when ctoprim
      // wrote it, so it covers grow(box,4) then
      R.qf_grow = B.internal_q ? 4 : qf_grow;
      take(L, grow(B.bx, R.qf_grow), nt, 4, R.qf, false, true);
      R.qf_in_prep = B.internal_q ? 0 : 1;
      add_slab_segs(L, K_PREP, (int)r, B.internal_q ? g1 : grow(B.bx, qf_grow), slabs, z0);
    } else {
      add_slab_segs(L, K_PREP, (int)r, g1, slabs, z0);
    }
    take(L, nodes(nodes(nodes(B.bx, 0), 1), 2), 1, 8, R.divu);
    for (int d = 0; d < 3; ++d) {
      IBox tb = g1;
      tb.hi[d] += 1;  // d-faces lo-1 .. hi+2
      take(L, tb, nt, L.esz, R.trm[d], true);
      take(L, tb, nt, L.esz, R.trp[d], true);
      sb[d] = g1;
      if (L.tile_trace) add_trace_tiles(L, (int)r, d, g1);
    }
    add_dir_segs(L, K_TRACE, (int)r, sb, slabs, z0);
    for (int d = 0; d < 3; ++d) {
      IBox fb = nodes(grow_dir(g1, d, -1), d);  // d-faces lo..hi+1, others grown by 1
      take(L, fb, nf, L.esz, R.fi[d], true);
      sb[d] = fb;
    }
    add_dir_segs(L, K_FLUX0, (int)r, sb, slabs, z0);
    for (int d = 0; d < 3; ++d) {
      for (int o = 0; o < 3; ++o) {
        if (o == d) continue;
        const int t = 3 - d - o;
        IBox b = nodes(B.bx, d);
        b = grow_dir(b, t, 1);
        take(L, b, nf, L.esz, R.fdo[d][o], true);
      }
      // one thread per d-face computes both (d|o) pairs that reach it
      sb[d] = nodes(grow_dir(g1, d, -1), d);
    }
    add_dir_segs(L, K_FLUX1, (int)r, sb, slabs, z0);
    // mixed form without flux export: FP32 final fluxes (FP64 accumulation in k_consup)
    R.ff_single = (single && !B.flx[0].p && !B.flx[1].p && !B.flx[2].p && !B.umeth) ? 1 : 0;
    const size_t fsz = R.ff_single ? 4 : 8;
    R.umeth = B.umeth ? 1 : 0;
    if (B.umeth) {
      L.umeth = 1;
      R.pdivu = B.pdivu;
    }
    for (int d = 0; d < 3; ++d) {
      const IBox fb = nodes(B.bx, d);
      // the mixed form's FP32 final fluxes are workspace arrays in the blocked layout; FP64
      // final fluxes (workspace or the caller's flux FABs) keep the Array4 layout
      if (B.flx[d].p) {
        R.ff[d] = B.flx[d];
      } else {
        take(L, fb, nv, fsz, R.ff[d], R.ff_single != 0);
      }
      if (B.umeth)
        R.qec[d] = B.qec[d];
      else
        take(L, fb, 2, fsz, R.qec[d], R.ff_single != 0);
      sb[d] = fb;
    }
    add_dir_segs(L, K_FLUX2, (int)r, sb, slabs, z0);
    // Source/Godunov.cpp:440-468: faces of the box on an inflow or user_bc domain
    // boundary get their final fluxes again from PLM states without transverse terms
    for (int d = 0; d < 3; ++d) {
      const bool lo_bc = (B.bclo[d] == PCG_BC_INFLOW || B.bclo[d] == PCG_BC_USER) && B.bx.lo[d] <= B.domlo[d];
      const bool hi_bc = (B.bchi[d] == PCG_BC_INFLOW || B.bchi[d] == PCG_BC_USER) && B.bx.hi[d] + 1 >= B.domhi[d] + 1;
      if (lo_bc) {
        IBox fb = nodes(B.bx, d);
        fb.hi[d] = B.domlo[d];
        if (fb.ok()) add_seg(L, K_LOWBC, (int)r, d, fb);
      }
      if (hi_bc) {
        IBox fb = nodes(B.bx, d);
        fb.lo[d] = B.domhi[d] + 1;
        if (fb.ok()) add_seg(L, K_LOWBC, (int)r, d, fb);
      }
    }
    add_seg(L, K_CONSUP, (int)r, 0, B.bx);
    L.regions.push_back(R);
  }
  // alternate traversal directions of successive stages (see add_dir_segs); K_CONSUP
  // keeps one segment per region in region order (the per-box timesteps index it)
  for (int st = K_CTOPRIM; st <= K_FLUX2; ++st)
    if ((kOrderReverseStages >> st) & 1u) reverse_segs(L, st);
}

void rebase(pcg::View& v, char* base) {
  v.p = base + reinterpret_cast<size_t>(v.p);
}

void rebase_workspace(Layout& L, const std::vector<BoxIn>& boxes, char* base) {
  for (size_t r = 0; r < L.regions.size(); ++r) {
    pcg::Region& R = L.regions[r];
    const BoxIn& B = boxes[r];
    if (B.internal_q) {
      if (L.esz != 4) rebase(R.q, base);  // FP64 forms only (see build_layout)
      rebase(R.qa, base);
    }
    rebase(R.prep, base);
    if (R.qf.p || L.esz == 4) rebase(R.qf, base);
    rebase(R.divu, base);
    for (int d = 0; d < 3; ++d) {
      rebase(R.trm[d], base);
      rebase(R.trp[d], base);
      rebase(R.fi[d], base);
      for (int o = 0; o < 3; ++o)
        if (o != d) rebase(R.fdo[d][o], base);
      if (!B.flx[d].p) rebase(R.ff[d], base);
      if (!B.umeth) rebase(R.qec[d], base);
    }
  }
}

// Device copy of the region and segment tables.
struct Tables {
  void* dev = nullptr;
  size_t bytes = 0;
  const pcg::Region* regions = nullptr;
  const pcg::Seg* segs[K_NKIND] = {};
  const void* tmaps = nullptr;  // tensor maps of the TMA-staged trace (3 per region)
  int32_t* err = nullptr;       // device error word
  bool maps_ok = false;         // every tensor map encoded
  std::vector<char> host;
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    cudaGetLastError();
  });
  return fn;
}

// The three tensor maps of a region's FP32 primitive copy qf (x fastest, then y, z,
// component), with the boxes of the x, y and z traces (pcg::trace_box_*): 40 x 4 x 1,
// 36 x 8 x 1 and 36 x 1 x 8 cells, every component.
bool encode_trace_maps(const pcg::Region& R, int nc, char* out) {
  PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
  if (!enc || !R.qf.p) return false;
  const uintptr_t base = reinterpret_cast<uintptr_t>(R.qf.p);
  if (base % 16 || R.qf.js % 4 || R.qf.blocked) return false;
  const cuuint64_t dims[4] = {cuuint64_t(R.qf.js), cuuint64_t(R.qf.ks / R.qf.js), cuuint64_t(R.qf.ns / R.qf.ks),
                              cuuint64_t(nc)};
  const cuuint64_t strides[3] = {cuuint64_t(R.qf.js) * 4, cuuint64_t(R.qf.ks) * 4, cuuint64_t(R.qf.ns) * 4};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  for (int d = 0; d < 3; ++d) {
    const cuuint32_t box[4] = {cuuint32_t(pcg::trace_box_x(d)), cuuint32_t(pcg::trace_box_y(d)),
                               cuuint32_t(pcg::trace_box_z(d)), cuuint32_t(nc)};
    CUtensorMap* m = reinterpret_cast<CUtensorMap*>(out + d * pcg::kTensorMapBytes);
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, reinterpret_cast<void*>(base), dims, strides,
                           box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
  }
  return true;
}

// encode = false: sizing only, before the workspace addresses exist (no tensor maps).
void pack_tables(const Layout& L, Tables& T, bool encode = true) {
  static_assert(sizeof(CUtensorMap) == pcg::kTensorMapBytes, "CUtensorMap size");
  size_t off = L.regions.size() * sizeof(pcg::Region);
  size_t seg_off[K_NKIND];
  for (int s = 0; s < K_NKIND; ++s) {
    off = (off + 15) / 16 * 16;
    seg_off[s] = off;
    off += L.segs[s].size() * sizeof(pcg::Seg);
  }
  off = (off + 127) / 128 * 128;  // tensor maps: 64-byte aligned (the table base is 256-aligned)
  const size_t map_off = off;
  if (L.tile_trace) off += L.regions.size() * 3 * pcg::kTensorMapBytes;
  const size_t err_off = off;
  off += 16;
  T.bytes = off;
  T.host.assign(T.bytes, 0);
  if (!L.regions.empty()) std::memcpy(T.host.data(), L.regions.data(), L.regions.size() * sizeof(pcg::Region));
  for (int s = 0; s < K_NKIND; ++s)
    if (!L.segs[s].empty()) std::memcpy(T.host.data() + seg_off[s], L.segs[s].data(), L.segs[s].size() * sizeof(pcg::Seg));
  T.maps_ok = L.tile_trace && encode;
  for (size_t r = 0; r < L.regions.size() && T.maps_ok; ++r)
    T.maps_ok = encode_trace_maps(L.regions[r], pcg::nt_comps(L.ns),
                                  T.host.data() + map_off + r * 3 * pcg::kTensorMapBytes);
  // device pointers are filled in by bind_tables once T.dev exists
  for (int s = 0; s < K_NKIND; ++s) T.segs[s] = reinterpret_cast<const pcg::Seg*>(seg_off[s]);
  T.tmaps = reinterpret_cast<const void*>(map_off);
  T.err = reinterpret_cast<int32_t*>(err_off);
}

void bind_tables(Tables& T) {
  char* base = static_cast<char*>(T.dev);
  T.regions = reinterpret_cast<const pcg::Region*>(base);
  T.tmaps = base + reinterpret_cast<size_t>(T.tmaps);
  T.err = reinterpret_cast<int32_t*>(base + reinterpret_cast<size_t>(T.err));
  for (int s = 0; s < K_NKIND; ++s) T.segs[s] = reinterpret_cast<const pcg::Seg*>(base + reinterpret_cast<size_t>(T.segs[s]));
}

// One launch of the kernel of `stage` over the segments of kind `segs` (launch variant var).
int launch_segs(const Layout& L, const Tables& T, const pcg_hydro_params* p, int stage, int segs, int var,
                const double* dt_dev, cudaStream_t s) {
  if (L.nblocks[segs] == 0) return PCG_OK;
  const bool single = p->precision_mode == PCG_PREC_MIXED;
  pcg::StageArgs a{};
  a.tmaps = T.tmaps;
  a.err = T.err;
  a.regions = T.regions;
  a.segs = T.segs[segs];
  a.nseg = (int32_t)L.segs[segs].size();
  a.ppm_type = p->ppm_type;
  a.plm_iorder = p->plm_iorder;
  a.use_flattening = p->use_flattening;
  a.use_hybrid_weno = p->use_hybrid_weno;
  a.weno_scheme = p->weno_scheme;
  a.umeth = L.umeth;
  a.difmag = p->difmag;
  a.dt_dev = dt_dev;
  cudaError_t e = (p->precision_mode == PCG_PREC_FP64)
                    ? pcg_strict::launch_stage(stage, L.ns, false, a, L.nblocks[segs], var, s)
                    : pcg_fast::launch_stage(stage, L.ns, single, a, L.nblocks[segs], var, s);
  if (e != cudaSuccess) return fail(PCG_ECUDA, "stage %d launch: %s", stage, cudaGetErrorString(e));
  return PCG_OK;
}

int launch_kind(const Layout& L, const Tables& T, const pcg_hydro_params* p, int kind, const double* dt_dev,
                cudaStream_t s) {
  int var = kind < K_NSTAGE ? variant_of(p->precision_mode, L.ns, kind) : 0;
  if (var >= kTileVariant) {
    var -= kTileVariant;
    // the mixed form's tiled trace (variants 3-5), when every tensor map was encoded
    if (kind == K_TRACE && L.tile_trace && T.maps_ok) kind = K_TRACE_TILE;
  }
  return launch_segs(L, T, p, kind, kind, var, dt_dev, s);
}

int launch_stages(const Layout& L, const Tables& T, const pcg_hydro_params* p, int first, int last,
                  const double* dt_dev, cudaStream_t s) {
  for (int st = first; st <= last; ++st) {
    int rc = launch_kind(L, T, p, st, dt_dev, s);
    if (rc == PCG_OK && st == K_FLUX2) rc = launch_kind(L, T, p, K_LOWBC, dt_dev, s);
    if (rc) return rc;
  }
  return PCG_OK;
}

// One-shot execution: stream-ordered workspace and tables, launches, stream-ordered free.
int run_once(const pcg_hydro_params* p, std::vector<BoxIn>& boxes, int first, int last, cudaStream_t s) {
  int rc = ensure_eos(p->nspec);
  if (rc) return rc;
  Layout L;
  build_layout(L, boxes, p);
  if (L.oversize) return fail(PCG_EINVAL, "a region needs workspace arrays of 2^31 elements or more: use smaller boxes");
  void* ws = nullptr;
  if (L.ws_bytes) CUDA_TRY(ws_alloc(&ws, L.ws_bytes, s));
  rebase_workspace(L, boxes, static_cast<char*>(ws));
  Tables T;
  pack_tables(L, T);
  cudaError_t e = ws_alloc(&T.dev, T.bytes, s);
  if (e != cudaSuccess) {
    if (ws) cudaFreeAsync(ws, s);
    cudaGetLastError();
    return fail(PCG_ENOMEM, "table allocation: %s", cudaGetErrorString(e));
  }
  e = upload(T.dev, T.host.data(), T.bytes, s);
  if (e == cudaSuccess) {
    bind_tables(T);
    rc = launch_stages(L, T, p, first, last, nullptr, s);
  } else {
    rc = fail(PCG_ECUDA, "table upload: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(T.dev, s);
  if (ws) cudaFreeAsync(ws, s);
  return rc;
}

int box_from_params(const pcg_hydro_params* p, const int32_t* lo, const int32_t* hi, BoxIn& B) {
  B = BoxIn{};
  B.bx = mkbox(lo, hi);
  for (int d = 0; d < 3; ++d) {
    B.domlo[d] = p->domlo[d];
    B.domhi[d] = p->domhi[d];
    B.bclo[d] = p->bclo[d];
    B.bchi[d] = p->bchi[d];
    B.dx[d] = p->dx[d];
  }
  B.dt = p->dt;
  return check_box_common(B.bx, B.dx, B.dt, B.bclo, B.bchi);
}

int box_from_desc(const pcg_box& b, int nv, BoxIn& B, bool need_uout = true) {
  B = BoxIn{};
  B.bx = mkbox(b.lo, b.hi);
  for (int d = 0; d < 3; ++d) {
    B.domlo[d] = b.domlo[d];
    B.domhi[d] = b.domhi[d];
    B.bclo[d] = b.bclo[d];
    B.bchi[d] = b.bchi[d];
    B.dx[d] = b.dx[d];
  }
  B.dt = b.dt;
  int rc = check_box_common(B.bx, B.dx, B.dt, B.bclo, B.bchi);
  if (rc) return rc;
  if ((rc = check_array("box uin", &b.uin, grow(B.bx, 4), nv))) return rc;
  if ((need_uout || b.uout.p) && (rc = check_array("box uout", &b.uout, B.bx, nv))) return rc;
  B.uin = view_of(&b.uin);
  B.uout = view_of(&b.uout);
  for (int d = 0; d < 3; ++d) {
    if (b.flx[d].p) {
      if ((rc = check_array("box flx", &b.flx[d], nodes(B.bx, d), nv))) return rc;
      B.flx[d] = view_of(&b.flx[d]);
    }
  }
  B.internal_q = true;
  B.zero_uout = true;
  return PCG_OK;
}

// Merge boxes that tile one shared array into their bounding box. Every output of the
// advance depends only on traced states in grow(box,1), whose flattening stencil
// (+-3) always lies inside the grow(box,4) FAB, so the result of a box does not
// depend on how its level is cut into boxes; a merged region gives bit-identical
// hydro sources and skips the halo work the separate boxes would repeat.
void fuse_boxes(std::vector<BoxIn>& boxes) {
  std::vector<bool> used(boxes.size(), false);
  std::vector<BoxIn> out;
  for (size_t a = 0; a < boxes.size(); ++a) {
    if (used[a]) continue;
    std::vector<size_t> grp{a};
    used[a] = true;
    const BoxIn& A = boxes[a];
    bool mergeable = !A.flx[0].p && !A.flx[1].p && !A.flx[2].p;
    for (size_t b = a + 1; mergeable && b < boxes.size(); ++b) {
      const BoxIn& B = boxes[b];
      if (used[b] || B.flx[0].p || B.flx[1].p || B.flx[2].p) continue;
      if (B.uin.p != A.uin.p || B.uout.p != A.uout.p || B.uin.js != A.uin.js || B.uin.ks != A.uin.ks ||
          B.uout.js != A.uout.js || B.uout.ks != A.uout.ks || B.dt != A.dt)
        continue;
      bool same = true;
      for (int d = 0; d < 3; ++d)
        same = same && B.dx[d] == A.dx[d] && B.domlo[d] == A.domlo[d] && B.domhi[d] == A.domhi[d] &&
               B.bclo[d] == A.bclo[d] && B.bchi[d] == A.bchi[d] && B.uin.b[d] == A.uin.b[d] &&
               B.uout.b[d] == A.uout.b[d];
      if (!same) continue;
      grp.push_back(b);
    }
    IBox bb = A.bx;
    int64_t vol = 0;
    for (size_t g : grp) {
      for (int d = 0; d < 3; ++d) {
        bb.lo[d] = std::min(bb.lo[d], boxes[g].bx.lo[d]);
        bb.hi[d] = std::max(bb.hi[d], boxes[g].bx.hi[d]);
      }
      vol += boxes[g].bx.cells();
    }
    bool disjoint = true;
    for (size_t x = 0; x < grp.size() && disjoint; ++x)
      for (size_t y = x + 1; y < grp.size() && disjoint; ++y) {
        const IBox &p = boxes[grp[x]].bx, &q = boxes[grp[y]].bx;
        bool ov = true;
        for (int d = 0; d < 3; ++d) ov = ov && p.lo[d] <= q.hi[d] && q.lo[d] <= p.hi[d];
        disjoint = !ov;
      }
    // the merged region's largest workspace array (QVAR components on grow(region, 4))
    // must stay addressable with 32-bit offsets
    const bool fits = grow(bb, 4).cells() * pcg::qvar(pcg::MAXNS) <= pcg::kMaxViewElems;
    if (grp.size() > 1 && disjoint && vol == bb.cells() && fits) {
      BoxIn M = A;
      M.bx = bb;
      out.push_back(M);
      for (size_t g : grp) used[g] = true;
    } else {
      out.push_back(A);
      for (size_t g = 1; g < grp.size(); ++g) used[grp[g]] = false;
    }
  }
  boxes.swap(out);
}

int aux_segments(const std::vector<IBox>& bx, std::vector<pcg::Seg>& segs, int64_t& nblocks) {
  segs.clear();
  nblocks = 0;
  for (size_t r = 0; r < bx.size(); ++r) {
    pcg::Seg s{};
    s.region = (int32_t)r;
    for (int d = 0; d < 3; ++d) { s.lo[d] = bx[r].lo[d]; s.n[d] = (int)bx[r].n(d); }
    s.count = bx[r].cells();
    s.blk0 = nblocks;
    segs.push_back(s);
    nblocks += (s.count + kThreads - 1) / kThreads;
  }
  return PCG_OK;
}

}  // namespace

// ====================================================================== C ABI
struct pcg_plan {
  pcg_hydro_params prm;
  std::vector<BoxIn> boxes;
  Layout L;
  Tables T;
  void* ws = nullptr;
  // auxiliary kernels over the original (unfused) boxes
  std::vector<pcg::AuxBox> aux;
  std::vector<pcg::Seg> aux_segs;
  int64_t aux_blocks = 0;
  void* aux_dev = nullptr;  // AuxBox[] + Seg[] + partial[]
  pcg::AuxBox* d_aux = nullptr;
  pcg::Seg* d_aux_segs = nullptr;
  double* d_partial = nullptr;
  int device = 0;
};

namespace pcg {
// The message pcg_last_error returns, set by the other host units (pcg_fluxreg.cu).
int set_error(int code, const char* msg) {
  g_err = msg;
  return code;
}
}  // namespace pcg

extern "C" {

int pcg_init(int device) {
  CUDA_TRY(cudaSetDevice(device));
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;  // keep freed workspace cached in the pool
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaGetLastError();
  return PCG_OK;
}

const char* pcg_last_error(void) { return g_err.c_str(); }

int pcg_set_eos_gamma(double gamma, double mw) {
  if (!(gamma > 1.0) || !(mw > 0.0)) return fail(PCG_EINVAL, "gamma must be > 1 and mw > 0");
  pcg::EosConst c{};
  c.kind = 0;
  c.nspec = 1;
  c.gamma = gamma;
  c.imw[0] = 1.0 / mw;
  c.gammaf = (float)gamma;
  c.imwf[0] = (float)c.imw[0];
  return store_eos(0, c);
}

int pcg_set_eos_nasa7(int nspec, const double* mw, const double* tmid, const double* a_lo, const double* a_hi) {
  if (nspec < 2 || nspec > pcg::MAXNS) return fail(PCG_EINVAL, "nspec must be in 2..%d", pcg::MAXNS);
  if (!species_built(nspec))
    return fail(PCG_EUNSUPPORTED, "nspec=%d: this build has kernels for %s species", nspec, species_list().c_str());
  if (!mw || !tmid || !a_lo || !a_hi) return fail(PCG_EINVAL, "NULL table");
  pcg::EosConst c{};
  c.kind = 1;
  c.nspec = nspec;
  c.uniform_tmid = 1;
  for (int k = 1; k < nspec; ++k)
    if (tmid[k] != tmid[0]) c.uniform_tmid = 0;
  for (int k = 0; k < nspec; ++k) {
    if (!(mw[k] > 0.0)) return fail(PCG_EINVAL, "mw[%d] must be > 0", k);
    const double rw = pcg::RU / mw[k];
    c.imw[k] = 1.0 / mw[k];
    c.tmid[k] = tmid[k];
    for (int r = 0; r < 2; ++r) {
      const double* a = (r == 0 ? a_lo : a_hi) + 7 * k;
      c.cvc[k][r][0] = rw * (a[0] - 1.0);
      c.cvc[k][r][1] = rw * a[1];
      c.cvc[k][r][2] = rw * a[2];
      c.cvc[k][r][3] = rw * a[3];
      c.cvc[k][r][4] = rw * a[4];
      c.ec[k][r][0] = rw * a[5];
      c.ec[k][r][1] = rw * (a[0] - 1.0);
      c.ec[k][r][2] = rw * (a[1] / 2.0);
      c.ec[k][r][3] = rw * (a[2] / 3.0);
      c.ec[k][r][4] = rw * (a[3] / 4.0);
      c.ec[k][r][5] = rw * (a[4] / 5.0);
      for (int i = 0; i < 5; ++i) c.cvcf[k][r][i] = c.cvp[r][i][k] = (float)c.cvc[k][r][i];
      for (int i = 0; i < 6; ++i) c.ecf[k][r][i] = c.ecp[r][i][k] = (float)c.ec[k][r][i];
    }
    c.imwf[k] = c.imwp[k] = (float)c.imw[k];
    c.tmidf[k] = (float)c.tmid[k];
  }
  return store_eos(1, c);
}

int pcg_species_counts(int32_t* counts, int32_t max_counts) {
  std::vector<int> v;
  for (const pcg::UnitEntry& u : pcg::unit_table().units)
    if (u.kind == pcg::UNIT_STRICT && species_built(u.ns)) v.push_back(u.ns);
  std::sort(v.begin(), v.end());
  for (int32_t k = 0; counts && k < max_counts && k < (int32_t)v.size(); ++k) counts[k] = v[k];
  return (int)v.size();
}

int pcg_ctoprim(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3], const pcg_array4* u,
                pcg_array4* q, pcg_array4* qaux, pcg_stream_t stream) {
  int rc = check_params(prm);
  if (rc) return rc;
  const IBox bx = mkbox(lo, hi);
  if (!bx.ok()) return fail(PCG_EINVAL, "empty box");
  const int nv = pcg::nvar(prm->nspec), nq = pcg::qvar(prm->nspec);
  if ((rc = check_array("u", u, bx, nv)) || (rc = check_array("q", q, bx, nq)) ||
      (rc = check_array("qaux", qaux, bx, pcg::NQAUX)))
    return rc;
  if ((rc = ensure_eos(prm->nspec))) return rc;
  // A one-region plan with only the ctoprim stage, on the caller's arrays.
  Layout L;
  L.ns = prm->nspec;
  pcg::Region R{};
  R.uin = view_of(u);
  R.q = view_of(q);
  R.qa = view_of(qaux);
  L.regions.push_back(R);
  add_seg(L, K_CTOPRIM, 0, 0, bx);
  Tables T;
  pack_tables(L, T);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  CUDA_TRY(ws_alloc(&T.dev, T.bytes, s));
  cudaError_t e = upload(T.dev, T.host.data(), T.bytes, s);
  if (e == cudaSuccess) {
    bind_tables(T);
    pcg_hydro_params p = *prm;
    p.precision_mode = PCG_PREC_FP64;
    rc = launch_stages(L, T, &p, K_CTOPRIM, K_CTOPRIM, nullptr, s);
  } else {
    rc = fail(PCG_ECUDA, "table upload: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(T.dev, s);
  return rc;
}

int pcg_umdrv(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3], const pcg_array4* uin,
              pcg_array4* uout, const pcg_array4* q, const pcg_array4* qaux, const pcg_array4* src_q,
              pcg_array4* flx, const pcg_array4* area, const pcg_array4* vol, pcg_stream_t stream) {
  int rc = check_params(prm);
  if (rc) return rc;
  std::vector<BoxIn> boxes(1);
  BoxIn& B = boxes[0];
  if ((rc = box_from_params(prm, lo, hi, B))) return rc;
  const int nv = pcg::nvar(prm->nspec), nq = pcg::qvar(prm->nspec);
  const IBox g4 = grow(B.bx, 4);
  if ((rc = check_array("uin", uin, grow(B.bx, 1), nv))) return rc;
  if ((rc = check_array("uout", uout, B.bx, nv))) return rc;
  if ((rc = check_array("q", q, g4, nq))) return rc;
  if ((rc = check_array("qaux", qaux, g4, pcg::NQAUX))) return rc;
  if (src_q && src_q->p && (rc = check_array("src_q", src_q, g4, nq))) return rc;
  if (!flx || !area || !vol) return fail(PCG_EINVAL, "flx, area and vol are required");
  for (int d = 0; d < 3; ++d) {
    if ((rc = check_array("flx", &flx[d], nodes(B.bx, d), nv))) return rc;
    if ((rc = check_array("area", &area[d], nodes(B.bx, d), 1))) return rc;
  }
  if ((rc = check_array("vol", vol, B.bx, 1))) return rc;
  B.uin = view_of(uin);
  B.uout = view_of(uout);
  B.q = view_of(q);
  B.qa = view_of(qaux);
  B.srcq = view_of(src_q);
  B.vol = view_of(vol);
  for (int d = 0; d < 3; ++d) {
    B.area[d] = view_of(&area[d]);
    B.flx[d] = view_of(&flx[d]);
  }
  B.internal_q = false;
  B.zero_uout = false;
  return run_once(prm, boxes, K_PREP, K_CONSUP, reinterpret_cast<cudaStream_t>(stream));
}

int pcg_umeth(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3], const pcg_array4* q,
              const pcg_array4* qaux, const pcg_array4* src_q, pcg_array4* flx, pcg_array4* qec,
              const pcg_array4* area, pcg_array4* pdivu, const pcg_array4* vol, pcg_stream_t stream) {
  int rc = check_params(prm);
  if (rc) return rc;
  std::vector<BoxIn> boxes(1);
  BoxIn& B = boxes[0];
  if ((rc = box_from_params(prm, lo, hi, B))) return rc;
  const int nv = pcg::nvar(prm->nspec), nq = pcg::qvar(prm->nspec);
  const IBox g4 = grow(B.bx, 4);
  if ((rc = check_array("q", q, g4, nq))) return rc;
  if ((rc = check_array("qaux", qaux, g4, pcg::NQAUX))) return rc;
  if (src_q && src_q->p && (rc = check_array("src_q", src_q, g4, nq))) return rc;
  if (!flx || !qec || !area || !pdivu || !vol) return fail(PCG_EINVAL, "flx, qec, area, pdivu and vol are required");
  for (int d = 0; d < 3; ++d) {
    if ((rc = check_array("flx", &flx[d], nodes(B.bx, d), nv))) return rc;
    if ((rc = check_array("qec", &qec[d], nodes(B.bx, d), pcg::NGDNV))) return rc;
    if ((rc = check_array("area", &area[d], nodes(B.bx, d), 1))) return rc;
  }
  if ((rc = check_array("pdivu", pdivu, B.bx, 1))) return rc;
  if ((rc = check_array("vol", vol, B.bx, 1))) return rc;
  B.q = view_of(q);
  B.qa = view_of(qaux);
  B.srcq = view_of(src_q);
  B.vol = view_of(vol);
  B.pdivu = view_of(pdivu);
  for (int d = 0; d < 3; ++d) {
    B.area[d] = view_of(&area[d]);
    B.flx[d] = view_of(&flx[d]);
    B.qec[d] = view_of(&qec[d]);
  }
  B.internal_q = false;
  B.zero_uout = false;
  B.umeth = true;
  return run_once(prm, boxes, K_PREP, K_CONSUP, reinterpret_cast<cudaStream_t>(stream));
}

int pcg_srctoprim(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3], const pcg_array4* q,
                  const pcg_array4* qaux, const pcg_array4* src, pcg_array4* srcq, pcg_stream_t stream) {
  int rc = check_params(prm);
  if (rc) return rc;
  const IBox bx = mkbox(lo, hi);
  if (!bx.ok()) return fail(PCG_EINVAL, "empty box");
  const int nv = pcg::nvar(prm->nspec), nq = pcg::qvar(prm->nspec);
  if ((rc = check_array("q", q, bx, nq)) || (rc = check_array("qaux", qaux, bx, pcg::NQAUX)) ||
      (rc = check_array("src", src, bx, nv)) || (rc = check_array("srcq", srcq, bx, nq)))
    return rc;
  // a one-region table with only the srctoprim launch, on the caller's arrays
  Layout L;
  L.ns = prm->nspec;
  pcg::Region R{};
  R.q = view_of(q);
  R.qa = view_of(qaux);
  R.src = view_of(src);
  R.srcq = view_of(srcq);
  L.regions.push_back(R);
  add_seg(L, K_SRCQ, 0, 0, bx);
  Tables T;
  pack_tables(L, T);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  CUDA_TRY(ws_alloc(&T.dev, T.bytes, s));
  cudaError_t e = upload(T.dev, T.host.data(), T.bytes, s);
  if (e == cudaSuccess) {
    bind_tables(T);
    pcg_hydro_params p = *prm;
    p.precision_mode = PCG_PREC_FP64;  // FP64 in every form, reference operation order
    rc = launch_kind(L, T, &p, K_SRCQ, nullptr, s);
  } else {
    rc = fail(PCG_ECUDA, "table upload: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(T.dev, s);
  return rc;
}

int pcg_hydro_box(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3], const pcg_array4* uin,
                  pcg_array4* uout, pcg_array4* flx, pcg_stream_t stream) {
  int rc = check_params(prm);
  if (rc) return rc;
  pcg_box b{};
  for (int d = 0; d < 3; ++d) {
    b.lo[d] = lo[d];
    b.hi[d] = hi[d];
    b.domlo[d] = prm->domlo[d];
    b.domhi[d] = prm->domhi[d];
    b.bclo[d] = prm->bclo[d];
    b.bchi[d] = prm->bchi[d];
    b.dx[d] = prm->dx[d];
  }
  b.dt = prm->dt;
  if (!uin || !uout) return fail(PCG_EINVAL, "uin and uout are required");
  b.uin = *uin;
  b.uout = *uout;
  if (flx)
    for (int d = 0; d < 3; ++d) b.flx[d] = flx[d];
  std::vector<BoxIn> boxes(1);
  if ((rc = box_from_desc(b, pcg::nvar(prm->nspec), boxes[0]))) return rc;
  return run_once(prm, boxes, K_CTOPRIM, K_CONSUP, reinterpret_cast<cudaStream_t>(stream));
}

int pcg_hydro_boxes(const pcg_hydro_params* prm, int32_t nbox, const pcg_box* boxes, pcg_stream_t stream) {
  int rc = check_params(prm);
  if (rc) return rc;
  if (nbox < 0 || (nbox > 0 && !boxes)) return fail(PCG_EINVAL, "bad box list");
  if (nbox == 0) return PCG_OK;
  std::vector<BoxIn> bs(nbox);
  for (int b = 0; b < nbox; ++b)
    if ((rc = box_from_desc(boxes[b], pcg::nvar(prm->nspec), bs[b]))) return rc;
  return run_once(prm, bs, K_CTOPRIM, K_CONSUP, reinterpret_cast<cudaStream_t>(stream));
}

int pcg_step_boxes(const pcg_hydro_params* prm, int32_t nbox, const pcg_box* boxes, int32_t fill_ghosts,
                   double cfl, const double* dt, double* dt_next, pcg_stream_t stream) {
  int rc = check_params(prm);
  if (rc) return rc;
  if (nbox < 0 || (nbox > 0 && !boxes) || (nbox > 0 && !dt_next)) return fail(PCG_EINVAL, "bad arguments");
  if (!(cfl > 0.0) || !std::isfinite(cfl)) return fail(PCG_EINVAL, "cfl must be positive");
  if (nbox == 0) return PCG_OK;
  if ((rc = ensure_eos(prm->nspec))) return rc;
  const int nv = pcg::nvar(prm->nspec);
  std::vector<BoxIn> bs(nbox);
  for (int b = 0; b < nbox; ++b)
    if ((rc = box_from_desc(boxes[b], nv, bs[b], false))) return rc;
  Layout L;
  build_layout(L, bs, prm);
  if (L.oversize) return fail(PCG_EINVAL, "a region needs workspace arrays of 2^31 elements or more: use smaller boxes");
  for (int b = 0; b < nbox; ++b) L.regions[b].dt_ptr = dt ? dt + b : nullptr;
  // ghost fill table: each box is its own domain (periodic where both its boundary types
  // are interior, zero-gradient elsewhere)
  std::vector<pcg::FillBox> fills;
  int64_t fill_blocks = 0;
  if (fill_ghosts) {
    for (int b = 0; b < nbox; ++b) {
      pcg::FillBox f{};
      f.state = bs[b].uin;
      int64_t inner = 1, outer = 1;
      for (int d = 0; d < 3; ++d) {
        f.dlo[d] = bs[b].bx.lo[d];
        f.dhi[d] = bs[b].bx.hi[d];
        if (bs[b].bclo[d] == PCG_BC_INTERIOR && bs[b].bchi[d] == PCG_BC_INTERIOR) f.periodic |= 1 << d;
        inner *= bs[b].bx.n(d);
        outer *= bs[b].bx.n(d) + 8;
      }
      f.count = outer - inner;
      f.blk0 = fill_blocks;
      fill_blocks += (f.count + kThreads - 1) / kThreads;
      fills.push_back(f);
    }
  }
  // one stream-ordered allocation: [workspace | tables | fill table | block minima]
  Tables T;
  pack_tables(L, T, false);
  const size_t off_t = (L.ws_bytes + kAlign - 1) / kAlign * kAlign;
  const size_t off_f = off_t + (T.bytes + kAlign - 1) / kAlign * kAlign;
  const size_t off_p = off_f + (fills.size() * sizeof(pcg::FillBox) + kAlign - 1) / kAlign * kAlign;
  const size_t total = off_p + size_t(std::max<int64_t>(L.nblocks[K_CONSUP], 1)) * sizeof(double);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  void* mem = nullptr;
  CUDA_TRY(ws_alloc(&mem, total, s));
  char* base = static_cast<char*>(mem);
  rebase_workspace(L, bs, base);
  Tables T2;
  pack_tables(L, T2);  // the regions now hold the workspace addresses
  T2.dev = base + off_t;
  std::vector<char> host(off_p - off_t, 0);
  std::memcpy(host.data(), T2.host.data(), T2.bytes);
  if (!fills.empty()) std::memcpy(host.data() + (off_f - off_t), fills.data(), fills.size() * sizeof(pcg::FillBox));
  cudaError_t e = upload(base + off_t, host.data(), host.size(), s);
  if (e != cudaSuccess) {
    cudaFreeAsync(mem, s);
    return fail(PCG_ECUDA, "table upload: %s", cudaGetErrorString(e));
  }
  bind_tables(T2);
  double* partial = reinterpret_cast<double*>(base + off_p);
  const bool strict = prm->precision_mode == PCG_PREC_FP64;
  if (fill_ghosts) {
    pcg::AuxArgs f{};
    f.fills = reinterpret_cast<const pcg::FillBox*>(base + off_f);
    f.nfill = nbox;
    f.ng = 4;
    f.ncomp = nv;
    e = pcg_strict::launch_aux(AUX_FILL_BOXES, prm->nspec, f, fill_blocks, s);
    if (e != cudaSuccess) rc = fail(PCG_ECUDA, "ghost fill: %s", cudaGetErrorString(e));
  }
  if (!rc) rc = launch_stages(L, T2, prm, K_CTOPRIM, K_FLUX2, nullptr, s);
  if (!rc) {
    pcg::StageArgs a{};
    a.regions = T2.regions;
    a.segs = T2.segs[K_CONSUP];
    a.nseg = (int32_t)L.segs[K_CONSUP].size();
    a.partial = partial;
    const int v = variant_of(prm->precision_mode, prm->nspec, K_CONSUP);
    e = strict ? pcg_strict::launch_advance(prm->nspec, a, L.nblocks[K_CONSUP], v, s)
               : pcg_fast::launch_advance(prm->nspec, a, L.nblocks[K_CONSUP], v, s);
    if (e == cudaSuccess) {
      pcg::AuxArgs r{};
      r.bsegs = T2.segs[K_CONSUP];
      r.partial = partial;
      r.cfl = cfl;
      r.dt_boxes = dt_next;
      e = pcg_strict::launch_aux(AUX_ESTDT_BOXES, prm->nspec, r, nbox, s);
    }
    if (e != cudaSuccess) rc = fail(PCG_ECUDA, "step tail: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(mem, s);
  return rc;
}

int pcg_hydro_workspace(const pcg_hydro_params* prm, int32_t nbox, const int32_t* lo, const int32_t* hi,
                        int64_t* bytes) {
  int rc = check_params(prm);
  if (rc) return rc;
  if (nbox < 0 || (nbox > 0 && (!lo || !hi)) || !bytes) return fail(PCG_EINVAL, "bad arguments");
  std::vector<BoxIn> bs(nbox);
  for (int b = 0; b < nbox; ++b) {
    bs[b] = BoxIn{};
    bs[b].bx = mkbox(lo + 3 * b, hi + 3 * b);
    if (bs[b].bx.cells() <= 0) return fail(PCG_EINVAL, "empty box %d", b);
    bs[b].internal_q = true;
  }
  Layout L;
  build_layout(L, bs, prm);
  if (L.oversize) return fail(PCG_EINVAL, "a region needs workspace arrays of 2^31 elements or more: use smaller boxes");
  Tables T;
  pack_tables(L, T, false);
  *bytes = int64_t(size_class((L.ws_bytes + kAlign - 1) / kAlign * kAlign + T.bytes));  // as ws_alloc takes it
  return PCG_OK;
}

int pcg_estdt(int32_t nspec, int32_t nbox, const pcg_box* boxes, double cfl, double* dt_out, pcg_stream_t stream) {
  if (!species_built(nspec))
    return fail(PCG_EUNSUPPORTED, "nspec=%d: this build has kernels for %s species", nspec, species_list().c_str());
  if (nbox <= 0 || !boxes || !dt_out) return fail(PCG_EINVAL, "bad arguments");
  int rc = ensure_eos(nspec);
  if (rc) return rc;
  std::vector<pcg::AuxBox> ab(nbox);
  std::vector<IBox> bx(nbox);
  for (int b = 0; b < nbox; ++b) {
    bx[b] = mkbox(boxes[b].lo, boxes[b].hi);
    if ((rc = check_array("uin", &boxes[b].uin, bx[b], pcg::nvar(nspec)))) return rc;
    ab[b] = pcg::AuxBox{};
    for (int d = 0; d < 3; ++d) { ab[b].lo[d] = bx[b].lo[d]; ab[b].hi[d] = bx[b].hi[d]; ab[b].dx[d] = boxes[b].dx[d]; }
    ab[b].uin = view_of(&boxes[b].uin);
  }
  std::vector<pcg::Seg> segs;
  int64_t nblocks = 0;
  aux_segments(bx, segs, nblocks);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const size_t b1 = nbox * sizeof(pcg::AuxBox), b2 = segs.size() * sizeof(pcg::Seg), b3 = nblocks * sizeof(double);
  std::vector<char> host(b1 + b2);
  std::memcpy(host.data(), ab.data(), b1);
  std::memcpy(host.data() + b1, segs.data(), b2);
  char* dev = nullptr;
  CUDA_TRY(ws_alloc(reinterpret_cast<void**>(&dev), b1 + b2 + b3, s));
  cudaError_t e = upload(dev, host.data(), b1 + b2, s);
  rc = PCG_OK;
  if (e == cudaSuccess) {
    pcg::AuxArgs a{};
    a.boxes = reinterpret_cast<const pcg::AuxBox*>(dev);
    a.segs = reinterpret_cast<const pcg::Seg*>(dev + b1);
    a.nseg = (int32_t)segs.size();
    a.partial = reinterpret_cast<double*>(dev + b1 + b2);
    a.npartial = nblocks;
    a.cfl = cfl;
    a.dt_out = dt_out;
    e = pcg_strict::launch_aux(AUX_ESTDT, nspec, a, nblocks, s);
    if (e == cudaSuccess) e = pcg_strict::launch_aux(AUX_ESTDT_FINAL, nspec, a, 1, s);
  }
  if (e != cudaSuccess) rc = fail(PCG_ECUDA, "estdt: %s", cudaGetErrorString(e));
  cudaFreeAsync(dev, s);
  return rc;
}

int pcg_update_state(int32_t nspec, int32_t nbox, const pcg_box* boxes, const pcg_array4* s_new, const double* dt,
                     pcg_stream_t stream) {
  if (!species_built(nspec))
    return fail(PCG_EUNSUPPORTED, "nspec=%d: this build has kernels for %s species", nspec, species_list().c_str());
  if (nbox <= 0 || !boxes || !s_new) return fail(PCG_EINVAL, "bad arguments");
  int rc = ensure_eos(nspec);
  if (rc) return rc;
  const int nv = pcg::nvar(nspec);
  std::vector<pcg::AuxBox> ab(nbox);
  std::vector<IBox> bx(nbox);
  for (int b = 0; b < nbox; ++b) {
    bx[b] = mkbox(boxes[b].lo, boxes[b].hi);
    if ((rc = check_array("uin", &boxes[b].uin, bx[b], nv)) || (rc = check_array("uout", &boxes[b].uout, bx[b], nv)) ||
        (rc = check_array("s_new", &s_new[b], bx[b], nv)))
      return rc;
    ab[b] = pcg::AuxBox{};
    for (int d = 0; d < 3; ++d) { ab[b].lo[d] = bx[b].lo[d]; ab[b].hi[d] = bx[b].hi[d]; ab[b].dx[d] = boxes[b].dx[d]; }
    ab[b].dt = boxes[b].dt;
    ab[b].uin = view_of(&boxes[b].uin);
    ab[b].uout = view_of(&boxes[b].uout);
    ab[b].snew = view_of(&s_new[b]);
  }
  std::vector<pcg::Seg> segs;
  int64_t nblocks = 0;
  aux_segments(bx, segs, nblocks);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const size_t b1 = nbox * sizeof(pcg::AuxBox), b2 = segs.size() * sizeof(pcg::Seg);
  std::vector<char> host(b1 + b2);
  std::memcpy(host.data(), ab.data(), b1);
  std::memcpy(host.data() + b1, segs.data(), b2);
  char* dev = nullptr;
  CUDA_TRY(ws_alloc(reinterpret_cast<void**>(&dev), b1 + b2, s));
  cudaError_t e = upload(dev, host.data(), b1 + b2, s);
  if (e == cudaSuccess) {
    pcg::AuxArgs a{};
    a.boxes = reinterpret_cast<const pcg::AuxBox*>(dev);
    a.segs = reinterpret_cast<const pcg::Seg*>(dev + b1);
    a.nseg = (int32_t)segs.size();
    a.dt_in = dt;
    e = pcg_strict::launch_aux(AUX_UPDATE, nspec, a, nblocks, s);
  }
  rc = (e == cudaSuccess) ? PCG_OK : fail(PCG_ECUDA, "update: %s", cudaGetErrorString(e));
  cudaFreeAsync(dev, s);
  return rc;
}

int pcg_fill_ghosts(const pcg_array4* state, const int32_t domlo[3], const int32_t domhi[3],
                    const int32_t periodic[3], int32_t ng, pcg_stream_t stream) {
  if (!state || !state->p || ng < 0) return fail(PCG_EINVAL, "bad arguments");
  IBox dom = mkbox(domlo, domhi);
  if (!dom.ok()) return fail(PCG_EINVAL, "empty domain");
  int rc = check_array("state", state, grow(dom, ng), 1);
  if (rc) return rc;
  for (int d = 0; d < 3; ++d)
    if (periodic[d] && dom.n(d) < ng) return fail(PCG_EINVAL, "periodic direction %d shorter than ng", d);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (ng == 0) return PCG_OK;
  pcg::AuxArgs a{};
  a.state = view_of(state);
  for (int e = 0; e < 3; ++e) { a.dlo[e] = domlo[e]; a.dhi[e] = domhi[e]; }
  a.ng = ng;
  a.periodic = (periodic[0] ? 1 : 0) | (periodic[1] ? 2 : 0) | (periodic[2] ? 4 : 0);
  a.ncomp = state->ncomp;
  const int64_t ncell = grow(dom, ng).cells() - dom.cells();  // every ghost cell, one thread each
  cudaError_t e = pcg_strict::launch_aux(AUX_FILL, 1, a, (ncell + kThreads - 1) / kThreads, s);
  if (e != cudaSuccess) return fail(PCG_ECUDA, "fill_ghosts: %s", cudaGetErrorString(e));
  return PCG_OK;
}

int pcg_copy_cells(const pcg_array4* src, const pcg_array4* dst, const int32_t lo[3], const int32_t hi[3],
                   pcg_stream_t stream) {
  if (!src || !dst || !src->p || !dst->p || !lo || !hi) return fail(PCG_EINVAL, "bad arguments");
  const IBox b = mkbox(lo, hi);
  if (!b.ok()) return fail(PCG_EINVAL, "empty box");
  if (src->ncomp != dst->ncomp) return fail(PCG_EINVAL, "component counts differ (%d, %d)", src->ncomp, dst->ncomp);
  int rc = check_array("src", src, b, src->ncomp);
  if (!rc) rc = check_array("dst", dst, b, dst->ncomp);
  if (rc) return rc;
  for (const pcg_array4* a : {src, dst})
    if (a->jstride < a->end[0] - a->begin[0] || a->kstride % a->jstride || a->kstride / a->jstride < a->end[1] - a->begin[1])
      return fail(PCG_EINVAL, "array rows must be contiguous with kstride a multiple of jstride");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // Both arrays in device memory: one kernel over all components (the packing and
  // unpacking of halo planes inside a captured step)
  cudaPointerAttributes pa{}, pb{};
  if (cudaPointerGetAttributes(&pa, src->p) == cudaSuccess && cudaPointerGetAttributes(&pb, dst->p) == cudaSuccess &&
      pa.type == cudaMemoryTypeDevice && pb.type == cudaMemoryTypeDevice && pa.device == pb.device) {
    pcg::AuxArgs a{};
    a.state = view_of(src);
    a.dst = view_of(dst);
    for (int d = 0; d < 3; ++d) {
      a.dlo[d] = lo[d];
      a.dhi[d] = hi[d];
    }
    a.ncomp = src->ncomp;
    const int64_t n = b.cells() * src->ncomp;
    const cudaError_t e = pcg_strict::launch_aux(AUX_COPY, 1, a, (n + kThreads - 1) / kThreads, s);
    return e == cudaSuccess ? PCG_OK : fail(PCG_ECUDA, "copy_cells: %s", cudaGetErrorString(e));
  }
  cudaGetLastError();
  // Whole rows in both arrays: each k-slice of the box is one contiguous run, so copy
  // slices rather than rows (host-to-device copies of short strided rows run at a
  // fraction of the bus bandwidth).
  const bool whole_rows = b.n(0) == src->jstride && b.n(0) == dst->jstride;
  for (int n = 0; n < src->ncomp && whole_rows; ++n) {
    const double* sp = src->p + n * src->nstride + (lo[1] - src->begin[1]) * src->jstride +
                       (int64_t)(lo[2] - src->begin[2]) * src->kstride;
    double* dp = dst->p + n * dst->nstride + (lo[1] - dst->begin[1]) * dst->jstride +
                 (int64_t)(lo[2] - dst->begin[2]) * dst->kstride;
    cudaError_t e = cudaMemcpy2DAsync(dp, (size_t)dst->kstride * sizeof(double), sp,
                                      (size_t)src->kstride * sizeof(double),
                                      (size_t)(b.n(1) * b.n(0)) * sizeof(double), (size_t)b.n(2), cudaMemcpyDefault, s);
    if (e != cudaSuccess) return fail(PCG_ECUDA, "copy_cells: %s", cudaGetErrorString(e));
  }
  if (whole_rows) return PCG_OK;
  for (int n = 0; n < src->ncomp; ++n) {
    cudaMemcpy3DParms c{};
    c.srcPtr = make_cudaPitchedPtr(src->p + n * src->nstride, (size_t)src->jstride * sizeof(double),
                                   (size_t)(src->end[0] - src->begin[0]), (size_t)(src->kstride / src->jstride));
    c.dstPtr = make_cudaPitchedPtr(dst->p + n * dst->nstride, (size_t)dst->jstride * sizeof(double),
                                   (size_t)(dst->end[0] - dst->begin[0]), (size_t)(dst->kstride / dst->jstride));
    c.srcPos = make_cudaPos((size_t)(lo[0] - src->begin[0]) * sizeof(double), (size_t)(lo[1] - src->begin[1]),
                            (size_t)(lo[2] - src->begin[2]));
    c.dstPos = make_cudaPos((size_t)(lo[0] - dst->begin[0]) * sizeof(double), (size_t)(lo[1] - dst->begin[1]),
                            (size_t)(lo[2] - dst->begin[2]));
    c.extent = make_cudaExtent((size_t)b.n(0) * sizeof(double), (size_t)b.n(1), (size_t)b.n(2));
    c.kind = cudaMemcpyDefault;
    cudaError_t e = cudaMemcpy3DAsync(&c, s);
    if (e != cudaSuccess) return fail(PCG_ECUDA, "copy_cells: %s", cudaGetErrorString(e));
  }
  return PCG_OK;
}

// ---- persistent plans ---------------------------------------------------------

int pcg_plan_create(const pcg_hydro_params* prm, int32_t nbox, const pcg_box* boxes, int32_t fuse, pcg_plan** out) {
  if (!out) return fail(PCG_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = check_params(prm);
  if (rc) return rc;
  if (nbox <= 0 || !boxes) return fail(PCG_EINVAL, "bad box list");
  if ((rc = ensure_eos(prm->nspec))) return rc;
  pcg_plan* P = new pcg_plan();
  P->prm = *prm;
  cudaGetDevice(&P->device);
  P->boxes.resize(nbox);
  for (int b = 0; b < nbox; ++b)
    if ((rc = box_from_desc(boxes[b], pcg::nvar(prm->nspec), P->boxes[b]))) {
      delete P;
      return rc;
    }
  // auxiliary tables over the boxes as given
  std::vector<IBox> bx(nbox);
  P->aux.resize(nbox);
  for (int b = 0; b < nbox; ++b) {
    bx[b] = P->boxes[b].bx;
    pcg::AuxBox& a = P->aux[b];
    a = pcg::AuxBox{};
    for (int d = 0; d < 3; ++d) { a.lo[d] = bx[b].lo[d]; a.hi[d] = bx[b].hi[d]; a.dx[d] = boxes[b].dx[d]; }
    a.dt = boxes[b].dt;
    a.uin = view_of(&boxes[b].uin);
    a.uout = view_of(&boxes[b].uout);
    a.snew = a.uin;  // in-place state update
  }
  aux_segments(bx, P->aux_segs, P->aux_blocks);
  if (fuse) fuse_boxes(P->boxes);
  build_layout(P->L, P->boxes, prm);
  if (P->L.oversize) {
    delete P;
    return fail(PCG_EINVAL, "a region needs workspace arrays of 2^31 elements or more: use smaller boxes or fuse = 0");
  }
  cudaError_t e = cudaSuccess;
  if (P->L.ws_bytes) e = cudaMalloc(&P->ws, P->L.ws_bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete P;
    return fail(PCG_ENOMEM, "workspace of %zu bytes: %s", P->L.ws_bytes, cudaGetErrorString(e));
  }
  rebase_workspace(P->L, P->boxes, static_cast<char*>(P->ws));
  pack_tables(P->L, P->T);
  const size_t b1 = P->aux.size() * sizeof(pcg::AuxBox), b2 = P->aux_segs.size() * sizeof(pcg::Seg),
               b3 = std::max<int64_t>(P->aux_blocks, P->L.nblocks[K_CONSUP]) * sizeof(double);
  if ((e = cudaMalloc(&P->T.dev, P->T.bytes)) == cudaSuccess &&
      (e = cudaMemcpy(P->T.dev, P->T.host.data(), P->T.bytes, cudaMemcpyHostToDevice)) == cudaSuccess &&
      (e = cudaMalloc(&P->aux_dev, b1 + b2 + b3)) == cudaSuccess) {
    char* d = static_cast<char*>(P->aux_dev);
    std::vector<char> host(b1 + b2);
    std::memcpy(host.data(), P->aux.data(), b1);
    std::memcpy(host.data() + b1, P->aux_segs.data(), b2);
    e = cudaMemcpy(d, host.data(), b1 + b2, cudaMemcpyHostToDevice);
    P->d_aux = reinterpret_cast<pcg::AuxBox*>(d);
    P->d_aux_segs = reinterpret_cast<pcg::Seg*>(d + b1);
    P->d_partial = reinterpret_cast<double*>(d + b1 + b2);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (P->ws) cudaFree(P->ws);
    if (P->T.dev) cudaFree(P->T.dev);
    if (P->aux_dev) cudaFree(P->aux_dev);
    delete P;
    return fail(PCG_ENOMEM, "plan tables: %s", cudaGetErrorString(e));
  }
  bind_tables(P->T);
  *out = P;
  return PCG_OK;
}

int pcg_plan_hydro(pcg_plan* P, const double* dt_dev, pcg_stream_t stream) {
  if (!P) return fail(PCG_EINVAL, "plan is NULL");
  int rc = ensure_eos(P->prm.nspec);
  if (rc) return rc;
  return launch_stages(P->L, P->T, &P->prm, K_CTOPRIM, K_CONSUP, dt_dev, reinterpret_cast<cudaStream_t>(stream));
}

int pcg_plan_stages(pcg_plan* P, int32_t first, int32_t last, const double* dt_dev, pcg_stream_t stream) {
  if (!P) return fail(PCG_EINVAL, "plan is NULL");
  if (first < 0 || last >= K_NSTAGE || first > last) return fail(PCG_EINVAL, "stage range %d..%d", first, last);
  int rc = ensure_eos(P->prm.nspec);
  if (rc) return rc;
  return launch_stages(P->L, P->T, &P->prm, first, last, dt_dev, reinterpret_cast<cudaStream_t>(stream));
}

int pcg_plan_estdt(pcg_plan* P, double cfl, double* dt_dev, pcg_stream_t stream) {
  if (!P || !dt_dev) return fail(PCG_EINVAL, "bad arguments");
  int rc = ensure_eos(P->prm.nspec);
  if (rc) return rc;
  pcg::AuxArgs a{};
  a.boxes = P->d_aux;
  a.segs = P->d_aux_segs;
  a.nseg = (int32_t)P->aux_segs.size();
  a.partial = P->d_partial;
  a.npartial = P->aux_blocks;
  a.cfl = cfl;
  a.dt_out = dt_dev;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = pcg_strict::launch_aux(AUX_ESTDT, P->prm.nspec, a, P->aux_blocks, s);
  if (e == cudaSuccess) e = pcg_strict::launch_aux(AUX_ESTDT_FINAL, P->prm.nspec, a, 1, s);
  return e == cudaSuccess ? PCG_OK : fail(PCG_ECUDA, "estdt: %s", cudaGetErrorString(e));
}

int pcg_plan_update(pcg_plan* P, const double* dt_dev, pcg_stream_t stream) {
  if (!P) return fail(PCG_EINVAL, "plan is NULL");
  int rc = ensure_eos(P->prm.nspec);
  if (rc) return rc;
  pcg::AuxArgs a{};
  a.boxes = P->d_aux;
  a.segs = P->d_aux_segs;
  a.nseg = (int32_t)P->aux_segs.size();
  a.dt_in = dt_dev;
  cudaError_t e = pcg_strict::launch_aux(AUX_UPDATE, P->prm.nspec, a, P->aux_blocks, reinterpret_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? PCG_OK : fail(PCG_ECUDA, "update: %s", cudaGetErrorString(e));
}

int pcg_plan_advance(pcg_plan* P, double cfl, const double* dt_dev, double* dt_next, pcg_stream_t stream) {
  if (!P || !dt_dev || !dt_next) return fail(PCG_EINVAL, "bad arguments");
  int rc = ensure_eos(P->prm.nspec);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if ((rc = launch_stages(P->L, P->T, &P->prm, K_CTOPRIM, K_FLUX2, dt_dev, s))) return rc;
  pcg::StageArgs a{};
  a.regions = P->T.regions;
  a.segs = P->T.segs[K_CONSUP];
  a.nseg = (int32_t)P->L.segs[K_CONSUP].size();
  a.dt_dev = dt_dev;
  a.partial = P->d_partial;
  const int64_t nb = P->L.nblocks[K_CONSUP];
  const int v = variant_of(P->prm.precision_mode, P->prm.nspec, K_CONSUP);
  cudaError_t e = (P->prm.precision_mode == PCG_PREC_FP64) ? pcg_strict::launch_advance(P->prm.nspec, a, nb, v, s)
                                                           : pcg_fast::launch_advance(P->prm.nspec, a, nb, v, s);
  if (e == cudaSuccess) {
    pcg::AuxArgs f{};
    f.partial = P->d_partial;
    f.npartial = nb;
    f.cfl = cfl;
    f.dt_out = dt_next;
    e = pcg_strict::launch_aux(AUX_ESTDT_FINAL, P->prm.nspec, f, 1, s);
  }
  return e == cudaSuccess ? PCG_OK : fail(PCG_ECUDA, "advance: %s", cudaGetErrorString(e));
}

int pcg_plan_info(const pcg_plan* P, int64_t* workspace_bytes, int32_t* nregions, int64_t* blocks_per_stage) {
  if (!P) return fail(PCG_EINVAL, "plan is NULL");
  if (workspace_bytes) *workspace_bytes = (int64_t)P->L.ws_bytes;
  if (nregions) *nregions = (int32_t)P->L.regions.size();
  if (blocks_per_stage) {
    for (int s = 0; s < K_NSTAGE; ++s) blocks_per_stage[s] = P->L.nblocks[s];
    blocks_per_stage[K_FLUX2] += P->L.nblocks[K_LOWBC];
  }
  return PCG_OK;
}

int pcg_trim_workspace(int32_t device, int64_t keep_bytes) {
  if (device < 0 || device >= kMaxDevices || keep_bytes < 0) return fail(PCG_EINVAL, "bad arguments");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[device]) return PCG_OK;
  const cudaError_t e = cudaMemPoolTrimTo(g_pool[device], size_t(keep_bytes));
  if (e != cudaSuccess) return fail(PCG_ECUDA, "pool trim: %s", cudaGetErrorString(e));
  return PCG_OK;
}

int pcg_reserve_workspace(int32_t device, int64_t bytes) {
  if (device < 0 || device >= kMaxDevices || bytes < 0) return fail(PCG_EINVAL, "bad arguments");
  if (bytes == 0) return PCG_OK;
  int cur = 0;
  CUDA_TRY(cudaGetDevice(&cur));
  CUDA_TRY(cudaSetDevice(device));
  // one allocation of `bytes` and its release: the pool keeps the memory (its release
  // threshold is unbounded), and later calls carve their workspace out of it
  cudaMemPool_t pool = nullptr;
  cudaStream_t s = nullptr;
  void* p = nullptr;
  cudaError_t e = workspace_pool(&pool);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    e = cudaMallocFromPoolAsync(&p, size_t(bytes), pool, s);
    if (e == cudaSuccess) e = cudaFreeAsync(p, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = e2;
    cudaStreamDestroy(s);
  }
  cudaSetDevice(cur);
  if (e != cudaSuccess) return fail(PCG_ECUDA, "workspace reservation of %lld bytes: %s", (long long)bytes,
                                    cudaGetErrorString(e));
  return PCG_OK;
}

int pcg_set_launch_variant(int32_t precision_mode, int32_t nspec, int32_t stage, int32_t variant) {
  if (precision_mode < 0 || precision_mode > 2 || !species_built(nspec) || stage < 0 || stage >= K_NSTAGE ||
      variant < 0 || variant > max_variant(precision_mode, stage))
    return fail(PCG_EINVAL, "launch variant (%d, %d, %d, %d) out of range", precision_mode, nspec, stage, variant);
  std::lock_guard<std::mutex> lk(g_var_mu);
  g_variant[precision_mode][nspec == 1 ? 0 : 1][stage] = variant;
  return PCG_OK;
}

int pcg_get_launch_variant(int32_t precision_mode, int32_t nspec, int32_t stage) {
  if (precision_mode < 0 || precision_mode > 2 || !species_built(nspec) || stage < 0 || stage >= K_NSTAGE)
    return fail(PCG_EINVAL, "launch variant query out of range");
  return variant_of(precision_mode, nspec, stage);
}

int pcg_plan_destroy(pcg_plan* P) {
  if (!P) return PCG_OK;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaSetDevice(P->device);
  if (P->ws) cudaFree(P->ws);
  if (P->T.dev) cudaFree(P->T.dev);
  if (P->aux_dev) cudaFree(P->aux_dev);
  cudaSetDevice(dev);
  cudaGetLastError();
  delete P;
  return PCG_OK;
}

}  // extern "C"

// ====================================================================== no-allocation entry
//
// pcg_hydro_box_noalloc is pcg_hydro_box for callers that must not allocate device
// memory. Inside a PeleC run the AMReX arena normally reserves most of the GPU's
// memory up front (amrex.the_arena_init_size), so a plugin's own cudaMalloc can fail or
// fragment what the arena left; other hosts run under a fixed memory budget or must not
// take the implicit device synchronisation of cudaMalloc/cudaFree in their step loop.
// This entry point keeps its launch tables and workspace in one statically sized device
// array of the library instead.
//
// * kNoAllocScratchBytes (32 MiB) is the whole budget: enough for a box of up to 21^3
//   cells with 9 species or 27^3 with one species in FP64 (27^3 / 34^3 in the mixed
//   form), without flux export. Larger boxes are rejected with PCG_EINVAL and a message
//   giving both sizes.
// * Every GPU that loads the library keeps the 32 MiB array until the process exits.
// * The array's device address comes from cudaGetSymbolAddress, once per device, on
//   the first call made with that device current (host code cannot use the symbol
//   itself: in host code it names a host-side stand-in). Make that first call outside
//   any stream capture.
// * All calls share the one array and it keeps the previous call's contents. Nothing in
//   it has to start at zero: the tables are copied in by each call and every stage
//   writes each workspace element before a later stage reads it. Calls that overlap on
//   the GPU (different streams, or different host threads without ordering) race on the
//   array; calls on one stream are ordered.
// * Nothing here calls cudaMalloc, cudaMallocAsync, cudaFree or any allocating library
//   routine. The tables travel with cudaMemcpyAsync from pageable host memory, which
//   stages them before the call returns.

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};

int noalloc_scratch(void** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(PCG_EINVAL, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p) return fail(PCG_ECUDA, "cudaGetSymbolAddress returned a null address");
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return PCG_OK;
}

}  // namespace

extern "C" int pcg_hydro_box_noalloc(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3],
                                     const pcg_array4* uin, pcg_array4* uout, pcg_array4* flx,
                                     pcg_stream_t stream) {
  int rc = check_params(prm);
  if (rc) return rc;
  if (!lo || !hi || !uin || !uout) return fail(PCG_EINVAL, "lo, hi, uin and uout are required");
  pcg_box b{};
  for (int d = 0; d < 3; ++d) {
    b.lo[d] = lo[d];
    b.hi[d] = hi[d];
    b.domlo[d] = prm->domlo[d];
    b.domhi[d] = prm->domhi[d];
    b.bclo[d] = prm->bclo[d];
    b.bchi[d] = prm->bchi[d];
    b.dx[d] = prm->dx[d];
  }
  b.dt = prm->dt;
  b.uin = *uin;
  b.uout = *uout;
  if (flx)
    for (int d = 0; d < 3; ++d) b.flx[d] = flx[d];
  std::vector<BoxIn> boxes(1);
  if ((rc = box_from_desc(b, pcg::nvar(prm->nspec), boxes[0]))) return rc;
  Layout L;
  build_layout(L, boxes, prm);
  if (L.oversize) return fail(PCG_EINVAL, "box too large");
  // scratch = [tables | workspace]; the table size does not depend on the addresses
  Tables T;
  pack_tables(L, T, false);
  const size_t ws_off = (T.bytes + kAlign - 1) / kAlign * kAlign;
  const size_t need = ws_off + L.ws_bytes;
  if (need > kNoAllocScratchBytes)
    return fail(PCG_EINVAL,
                "box [%d,%d,%d]-[%d,%d,%d] needs %zu bytes of scratch; pcg_hydro_box_noalloc has %zu "
                "(use pcg_hydro_box)",
                lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], need, kNoAllocScratchBytes);
  if ((rc = ensure_eos(prm->nspec))) return rc;
  void* base = nullptr;
  if ((rc = noalloc_scratch(&base))) return rc;
  char* scratch = static_cast<char*>(base);
  rebase_workspace(L, boxes, scratch + ws_off);
  Tables T2;
  pack_tables(L, T2);  // regions now hold the scratch addresses
  T2.dev = scratch;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemcpyAsync(T2.dev, T2.host.data(), T2.bytes, cudaMemcpyHostToDevice, s));
  bind_tables(T2);
  return launch_stages(L, T2, prm, K_CTOPRIM, K_CONSUP, nullptr, s);
}
