/*
 * pcg_hydro.h -- C ABI of the B200 (sm_100a) Godunov hydro advance.
 *
 * Drop-in for PeleC's unsplit Godunov path:
 *   PeleC::construct_hydro_source  (Source/Hydro.cpp:4-301, Source/PeleC.H:340)
 *     -> pc_ctoprim                (Source/Hydro.cpp:104-116, Source/PeleCUtilities.H:242-320)
 *     -> pc_umdrv                  (Source/Hydro.cpp:304-377, declared Source/Hydro.H:910-935)
 *        -> pc_umeth_3D            (Source/Godunov.cpp:59-476, declared Source/Godunov.H:1142-1162)
 *   PeleC::estTimeStep hydro part  (Source/PeleC.cpp:829-960, Source/Timestep.H:51-88)
 *   construct_Snew + computeTemp   (Source/Advance.cpp:397-417, Source/PeleC.cpp:2289-2305)
 *
 * Arrays are described by pcg_array4, which addresses memory exactly like
 * amrex::Array4<Real>: p[(i-begin[0]) + (j-begin[1])*jstride + (k-begin[2])*kstride
 * + n*nstride], end[] exclusive. All array pointers are DEVICE pointers unless stated.
 * Component layouts follow Source/IndexDefines.H (URHO..UTEMP, UFS; QRHO..QTEMP, QFS;
 * QGAMC..QRSPEC) with NUM_ADV = NUM_AUX = NUM_LIN = 0.
 *
 * Every call is asynchronous on the given stream (NULL = legacy default stream) and
 * returns PCG_OK or a negative PCG_E* code; pcg_last_error() gives the message of the
 * calling thread's last failure. Nothing aborts the process. Calls may be made from
 * several host threads at once (argument checks, plans and workspace are per call;
 * the shared tables are locked), with one exception: the EOS tables live in device
 * constant memory, one per species count, and pcg_set_eos_* replaces them with a
 * synchronous copy that is NOT ordered with kernels already queued on other streams.
 * Set the EOS once per run before advancing, or synchronise every stream that runs
 * this library's kernels before setting it again.
 */
#ifndef PCG_HYDRO_H
#define PCG_HYDRO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* pcg_stream_t; /* same type as cudaStream_t */

enum {
  PCG_OK = 0,
  PCG_EINVAL = -1,       /* bad argument (box, array extent, parameter) */
  PCG_ECUDA = -2,        /* a CUDA runtime call failed */
  PCG_ENOMEM = -3,       /* device allocation failed */
  PCG_EUNSUPPORTED = -4, /* option not implemented (a species count this build has no kernels for) */
  PCG_ETIMEDOUT = -5,    /* a bounded device wait gave up */
  PCG_EBUDGET = -6,      /* serving: request exceeds the memory budget */
  PCG_ENOEOS = -7        /* no EOS table set for this species count */
};

/* Physical boundary types, numbered as PCPhysBCType (Source/PeleC.H:49-57). */
enum { PCG_BC_INTERIOR = 0, PCG_BC_INFLOW, PCG_BC_OUTFLOW, PCG_BC_SYMMETRY,
       PCG_BC_SLIP_WALL, PCG_BC_NO_SLIP_WALL, PCG_BC_USER };

/* Arithmetic of the advance. */
enum {
  PCG_PREC_FP64 = 0,      /* plain FP64, reference operation order, no FMA contraction */
  PCG_PREC_FP64_FAST = 1, /* FP64 with FMA contraction */
  PCG_PREC_MIXED = 2      /* FP32 trace, Riemann and transverse terms; FP64 state,
                             flux-divergence accumulation, T(e) Newton and dt */
};

typedef struct pcg_array4 {
  double* p;
  int64_t jstride, kstride, nstride;
  int32_t begin[3], end[3];
  int32_t ncomp;
} pcg_array4;

/* Runtime parameters of pc_umdrv / pc_umeth_3D (names and defaults of
 * Source/Params/_cpp_parameters: difmag 0.1, ppm_type 0, plm_iorder 4,
 * use_flattening 1, use_hybrid_weno 0). */
typedef struct pcg_hydro_params {
  double dx[3];
  double dt;
  double difmag;
  int32_t ppm_type;       /* 0 PLM, 1 PPM */
  int32_t plm_iorder;     /* 1, 2 or 4 */
  int32_t use_flattening;
  int32_t use_hybrid_weno; /* 1: hybrid WENO edge values in the PPM trace (ppm_type 1) */
  int32_t weno_scheme;     /* with use_hybrid_weno: 0 WENO-JS5, 1 WENO-Z5, 2 WENO-Z7, 3 WENO-Z3 */
  int32_t domlo[3], domhi[3];
  int32_t bclo[3], bchi[3];
  int32_t nspec;          /* NUM_SPECIES: 1 (gamma law) or a mixture count of the build (pcg_species_counts) */
  int32_t precision_mode; /* PCG_PREC_* */
} pcg_hydro_params;

/* One box of a batched advance (the body of the MFIter loop, Source/Hydro.cpp:70-288).
 * uin: conserved state with >= 4 ghost cells; uout: hydro_source on the valid box
 * (overwritten: the batched call zeroes it first, as Hydro.cpp:47 does);
 * flx[d]: optional (p == NULL) area-weighted fluxes on the d-faces of the box.
 * dx, dt, domain and boundary data are per box so that boxes of unrelated runs can
 * share one launch. */
typedef struct pcg_box {
  int32_t lo[3], hi[3];
  int32_t domlo[3], domhi[3];
  int32_t bclo[3], bchi[3];
  double dx[3];
  double dt;
  pcg_array4 uin;
  pcg_array4 uout;
  pcg_array4 flx[3];
} pcg_box;

/* ---- set-up --------------------------------------------------------------- */

/* Select the CUDA device for the calling thread's subsequent calls. */
int pcg_init(int device);

/* EOS tables (PelePhysics' eos(), not in the reference checkout; documented
 * restatement). Gamma law: one species, constant gamma, molecular weight mw. */
int pcg_set_eos_gamma(double gamma, double mw);
/* Ideal-gas mixture with NASA-7 polynomials: a_lo/a_hi hold 7 coefficients per
 * species (HOST pointers), tmid the range split per species. nspec: 2 or more, one of
 * the build's species counts (PCG_EUNSUPPORTED otherwise). One mixture table is active
 * at a time. */
int pcg_set_eos_nasa7(int nspec, const double* mw, const double* tmid,
                      const double* a_lo, const double* a_hi);
/* The species counts this build has kernels for. The reference's NUM_SPECIES is a
 * compile-time constant of its mechanism (Source/IndexDefines.H:50-89); the library is
 * compiled for a list of them (particleclem_b200/build.py, PCG_NSPEC; 1 is the gamma
 * law). Writes up to max_counts of them, ascending, into counts (which may be NULL)
 * and returns how many there are. Host only: no device is touched. */
int pcg_species_counts(int32_t* counts, int32_t max_counts);

const char* pcg_last_error(void);

/* ---- the reference operator surface ---------------------------------------- */

/* pc_ctoprim over [lo,hi] (Source/PeleCUtilities.H:242-320): u -> q (QVAR comps),
 * qaux (NQAUX comps). Replaces the launch at Source/Hydro.cpp:104-116. */
int pcg_ctoprim(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3],
                const pcg_array4* u, pcg_array4* q, pcg_array4* qaux, pcg_stream_t stream);

/* pc_umdrv (Source/Hydro.H:910-935). q, qaux, src_q must cover grow(bx,4); src_q may
 * be NULL (no sources). uout is accumulated into (uout += hydro source), flx[3] is
 * overwritten with area-weighted fluxes, area[3]/vol are the geometry FABs.
 * Replaces Source/Hydro.cpp:245-249. */
int pcg_umdrv(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3],
              const pcg_array4* uin, pcg_array4* uout, const pcg_array4* q,
              const pcg_array4* qaux, const pcg_array4* src_q, pcg_array4* flx,
              const pcg_array4* area, const pcg_array4* vol, pcg_stream_t stream);

/* pc_srctoprim over [lo,hi] (Source/Hydro.H:14-68): the primitive-variable sources
 * srcq (QVAR comps) from the conserved sources src (NVAR comps, PeleC's
 * sources_for_hydro) and q, qaux. Replaces the launch at Source/Hydro.cpp:161-174; call
 * it over grow(bx,4) to feed pcg_umdrv / pcg_umeth. Always FP64 (reference order). */
int pcg_srctoprim(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3],
                  const pcg_array4* q, const pcg_array4* qaux, const pcg_array4* src,
                  pcg_array4* srcq, pcg_stream_t stream);

/* pc_umeth_3D on its own (Source/Godunov.cpp:59-476, declared Source/Godunov.H:1142-1162):
 * from q, qaux and src_q on grow(bx,4) (src_q may be NULL: no sources), flx[d] receives
 * the Godunov fluxes on the d-faces of bx as pc_umeth_3D leaves them (before the
 * artificial viscosity, species normalisation and area weighting of pc_adjust_fluxes;
 * component UTEMP is not written), qec[d] (NGDNV = 6 comps) the face states GDU, GDV, GDW,
 * GDPRES, GDGAME (GDRHO is not written, as in the reference), and pdivu the p div u of
 * Source/Godunov.H:1033-1060 on bx. area[3] and vol are the geometry FABs. */
int pcg_umeth(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3],
              const pcg_array4* q, const pcg_array4* qaux, const pcg_array4* src_q,
              pcg_array4* flx, pcg_array4* qec, const pcg_array4* area, pcg_array4* pdivu,
              const pcg_array4* vol, pcg_stream_t stream);

/* One construct_hydro_source box iteration (Source/Hydro.cpp:70-249 for a regular
 * box, no sources): ctoprim on grow(bx,4), then pc_umdrv. uout is zeroed first;
 * flx may be NULL. Geometry is uniform Cartesian from prm->dx. */
int pcg_hydro_box(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3],
                  const pcg_array4* uin, pcg_array4* uout, pcg_array4* flx,
                  pcg_stream_t stream);

/* pcg_hydro_box for callers that must not allocate device memory. No counterpart in
 * the reference: PeleC's own path allocates its temporaries from the AMReX arena. In a
 * GPU PeleC run that arena reserves most of the device memory at start-up, so a
 * plugin's cudaMalloc can fail or fragment what is left, and some hosts forbid the
 * synchronisation cudaMalloc/cudaFree imply inside their step loop. This entry keeps
 * its tables and workspace in one 32 MiB static device array of the library and
 * calls no allocator. Limit, without flux export: boxes up to 21^3 cells with 9 species
 * or 27^3 with one species in FP64 (27^3 / 34^3 in the mixed form; a little more with
 * flux export, whose fluxes live in the caller's arrays); larger boxes return
 * PCG_EINVAL. The array's
 * address is looked up on the first call per device: make that call outside any
 * stream capture. All calls share the array, so calls that overlap on the GPU
 * (different streams or unordered host threads) race; calls on one stream do not. */
int pcg_hydro_box_noalloc(const pcg_hydro_params* prm, const int32_t lo[3], const int32_t hi[3],
                          const pcg_array4* uin, pcg_array4* uout, pcg_array4* flx,
                          pcg_stream_t stream);

/* ---- batched form -------------------------------------------------------------- */

/* construct_hydro_source over many boxes in one set of launches: every box of the
 * list is advanced by its own dx/dt/domain/BCs; ppm_type, plm_iorder,
 * use_flattening, difmag, nspec and precision_mode come from prm (its dx, dt, dom*,
 * bc* are ignored). Uniform Cartesian geometry. */
int pcg_hydro_boxes(const pcg_hydro_params* prm, int32_t nbox, const pcg_box* boxes,
                    pcg_stream_t stream);

/* One full step of every box of a list of independent patches, each with its own
 * timestep: the step PeleC's level advance takes around construct_hydro_source
 * (Source/Advance.cpp:266-352) for a patch that is its own domain. Per box, in one set of
 * launches over all boxes: with fill_ghosts != 0, the ghost cells of boxes[b].uin (4
 * layers) from its own valid cells (periodic in a direction whose two boundary types are
 * PCG_BC_INTERIOR, zero-gradient otherwise); the hydro stages with timestep dt[b]
 * (dt: DEVICE array of nbox; NULL: boxes[b].dt); then S_new = S_old + dt hydro_source
 * with computeTemp, written over boxes[b].uin (the hydro source itself is not stored;
 * boxes[b].uout may be NULL); and dt_next[b] (DEVICE array of nbox) = cfl * the CFL
 * minimum of the box's new state (Source/Timestep.H:51-88), its next timestep.
 * Workspace as pcg_hydro_boxes. No counterpart in the reference (the serving loop of this
 * library advances ensemble patches with it). */
int pcg_step_boxes(const pcg_hydro_params* prm, int32_t nbox, const pcg_box* boxes, int32_t fill_ghosts,
                   double cfl, const double* dt, double* dt_next, pcg_stream_t stream);

/* Device bytes a pcg_hydro_boxes call over boxes [lo[3b], hi[3b]] (b < nbox) allocates
 * for its workspace and launch tables (stream-ordered, freed when the call's work
 * ends): the admission estimate of a serving loop under an HBM budget. Host only.
 * No counterpart in the reference (its temporaries come from the AMReX arena). */
int pcg_hydro_workspace(const pcg_hydro_params* prm, int32_t nbox, const int32_t* lo, const int32_t* hi,
                        int64_t* bytes);

/* pc_estdt_hydro over the valid cells of every box (Source/Timestep.H:51-88), the
 * min over boxes, times cfl (Source/PeleC.cpp:930). dt_out is a DEVICE pointer
 * to one double, written asynchronously. Each box's dx is used. */
int pcg_estdt(int32_t nspec, int32_t nbox, const pcg_box* boxes, double cfl,
              double* dt_out, pcg_stream_t stream);

/* construct_Snew (S_new = S_old + dt*hydro_source, Source/Advance.cpp:397-417) and
 * computeTemp (Source/PeleC.cpp:2289-2305: pc_rst_int_e default branch, then the
 * T(e) Newton of pc_cmpTemp) on the valid cells of every box: reads boxes[b].uin as
 * S_old and boxes[b].uout as hydro_source, writes S_new into s_new[b]. dt is a
 * DEVICE pointer (NULL: each box's dt). s_new may alias uin. */
int pcg_update_state(int32_t nspec, int32_t nbox, const pcg_box* boxes,
                     const pcg_array4* s_new, const double* dt, pcg_stream_t stream);

/* Single-level ghost fill of a domain-sized FAB covering grow(domain, ng): periodic
 * wrap in periodic directions, zero-gradient extrapolation (foextrap) otherwise.
 * The FillBoundary/FillPatch step that precedes the advance (Source/Advance.cpp:307-309). */
int pcg_fill_ghosts(const pcg_array4* state, const int32_t domlo[3], const int32_t domhi[3],
                    const int32_t periodic[3], int32_t ng, pcg_stream_t stream);

/* Copy the cells [lo, hi] of every component from src to dst, two arrays of equal
 * component count whose rows are contiguous (kstride a multiple of jstride); either may
 * be host or device memory (unified addressing tells which; pinned host memory for an
 * asynchronous copy). Between two arrays on one device: one kernel over all components;
 * otherwise one strided copy per component. Enqueued on stream. This moves a
 * level's valid cells between a host FAB and the device FAB whose ghost cells
 * pcg_fill_ghosts forms, so ghost cells do not cross the bus. No counterpart in the
 * reference (AMReX moves a MultiFab's valid region with its own copy routines). */
int pcg_copy_cells(const pcg_array4* src, const pcg_array4* dst, const int32_t lo[3], const int32_t hi[3],
                   pcg_stream_t stream);

/* ---- persistent plans (repeated steps, CUDA-graph capture) -------------------- */

/* A plan fixes a box list and owns its workspace and launch tables, so that its run
 * functions allocate nothing and can be captured in a CUDA graph. It replaces the
 * per-step box loop of construct_hydro_source (Source/Hydro.cpp:70-288) plus the
 * estTimeStep reduction and the state update of the level advance.
 * fuse != 0 lets the plan advance boxes that tile one shared state array as their
 * bounding box (bit-identical results, no repeated halo work). */
typedef struct pcg_plan pcg_plan;
int pcg_plan_create(const pcg_hydro_params* prm, int32_t nbox, const pcg_box* boxes,
                    int32_t fuse, pcg_plan** plan);
/* construct_hydro_source over the plan's boxes; dt_dev: DEVICE pointer to the step's
 * dt, or NULL to use each box's dt. */
int pcg_plan_hydro(pcg_plan* plan, const double* dt_dev, pcg_stream_t stream);
/* Stages first..last of pcg_plan_hydro only (0 ctoprim, 1 prep, 2 trace, 3 first
 * Riemann, 4 transverse Riemann, 5 final Riemann and flux adjustment, 6 consup), for
 * per-stage timing. */
int pcg_plan_stages(pcg_plan* plan, int32_t first, int32_t last, const double* dt_dev,
                    pcg_stream_t stream);
/* cfl * min over the plan's boxes of pc_estdt_hydro, into *dt_dev (DEVICE). */
int pcg_plan_estdt(pcg_plan* plan, double cfl, double* dt_dev, pcg_stream_t stream);
/* S_new = S_old + dt * hydro_source in place in each box's uin, then computeTemp. */
int pcg_plan_update(pcg_plan* plan, const double* dt_dev, pcg_stream_t stream);
/* One level step after the ghost fill with timestep *dt_dev (device): the hydro stages,
 * then in one pass per cell the flux divergence, S_new = S_old + dt * hydro_source with
 * computeTemp (in place in each box's uin) and the CFL minimum of S_new; *dt_next
 * (device, may equal dt_dev) receives cfl * that minimum, the next step's timestep
 * (PeleC's estTimeStep at the start of the next step, Source/PeleC.cpp:829-960, reads the
 * same valid cells). The hydro source arrays (uout) are not written. Same results as
 * pcg_plan_hydro + pcg_plan_update followed by pcg_plan_estdt. */
int pcg_plan_advance(pcg_plan* plan, double cfl, const double* dt_dev, double* dt_next, pcg_stream_t stream);
int pcg_plan_info(const pcg_plan* plan, int64_t* workspace_bytes, int32_t* nregions,
                  int64_t* blocks_per_stage /* [7] */);
int pcg_plan_destroy(pcg_plan* plan);

/* One-shot calls take their workspace stream-ordered from a memory pool the library
 * keeps per device without returning freed memory to the driver between calls. This
 * returns all but keep_bytes of the pool of CUDA device `device` to the driver (after
 * the work that used it completes). No counterpart in the reference. */
int pcg_trim_workspace(int32_t device, int64_t keep_bytes);
/* Grows that pool to hold at least `bytes` (one allocation and its release; returns when
 * done): a loop of one-shot calls whose workspace sizes vary (a serving loop) then takes
 * its workspace from memory the pool holds, where the first call of each new size would
 * otherwise wait for the driver to map memory (tens to hundreds of milliseconds
 * measured on B200). No counterpart in the reference. */
int pcg_reserve_workspace(int32_t device, int64_t bytes);

/* ---- coarse/fine: flux register, reflux, average-down ---------------------------- */

/* The coarse/fine use of the exported fluxes (Source/Hydro.cpp:281-287 ->
 * PeleC::update_flux_registers, Source/PeleC.cpp:1343-1400; PeleC::reflux,
 * Source/PeleC.cpp:1403-1414; the register class is AMReX's EBFluxRegister on regular
 * boxes, whose CrseAdd / FineAdd / Reflux these calls replace). A register sits between
 * a coarse level (domain crse_domlo..crse_domhi, periodic[d] != 0 where periodic) and
 * the fine boxes above it (fine index space, refinement ratio `ratio` in every
 * direction, boxes aligned to the ratio, inside the coarse domain, disjoint). It holds
 * one accumulator of ncomp doubles per coarse face on the coarse/fine boundary (faces on
 * non-periodic domain boundaries and between fine boxes have none). All calls are on the
 * device current at creation (a call with another device current returns PCG_EINVAL);
 * the register owns its device memory. */
typedef struct pcg_fluxreg pcg_fluxreg;
int pcg_fluxreg_create(int32_t ncomp, const int32_t crse_domlo[3], const int32_t crse_domhi[3],
                       const int32_t periodic[3], int32_t ratio, int32_t nfine, const int32_t* fine_lo /*[3*nfine]*/,
                       const int32_t* fine_hi /*[3*nfine]*/, pcg_fluxreg** out);
/* nfaces: accumulators (coarse/fine faces); ncells: coarse cells they correct. Host only. */
int pcg_fluxreg_info(const pcg_fluxreg* reg, int32_t* nfaces, int32_t* ncells);
/* Zero the accumulators (start of the coarse step, Source/Advance.cpp:30-31). */
int pcg_fluxreg_reset(pcg_fluxreg* reg, pcg_stream_t stream);
/* CrseAdd: coarse box [lo, hi] with its area-weighted fluxes flx[3] (the flx export of
 * pcg_box / pcg_hydro_box, d-faces lo..hi+1) of a step of dt: every register face of a
 * coarse cell in the box takes -s * dt * F (s = +1 on the cell's low face, -1 on its
 * high face). */
int pcg_fluxreg_crse_add(pcg_fluxreg* reg, const int32_t lo[3], const int32_t hi[3], const pcg_array4* flx /*[3]*/,
                         double dt, pcg_stream_t stream);
/* FineAdd: fine box [lo, hi] (one of the register's) with its area-weighted fluxes of a
 * fine step of dt: every register face it borders takes +s * dt * (the sum of its ratio^2
 * fine faces). Called once per fine box and fine substep. */
int pcg_fluxreg_fine_add(pcg_fluxreg* reg, const int32_t lo[3], const int32_t hi[3], const pcg_array4* flx /*[3]*/,
                         double dt, pcg_stream_t stream);
/* Reflux: S += (sum of the cell's accumulators) / vol on every coarse cell next to the
 * fine region (vol: the coarse cell volume). The caller recomputes T afterwards, as
 * PeleC's post_timestep does. */
int pcg_fluxreg_reflux(pcg_fluxreg* reg, pcg_array4* s_crse, double vol, pcg_stream_t stream);
int pcg_fluxreg_destroy(pcg_fluxreg* reg);
/* avgDown on regular boxes (PeleC::avgDown, Source/PeleC.cpp:1440, called at :1098;
 * AMReX's average_down): every coarse cell under the fine box [fine_lo, fine_hi] becomes the mean
 * of its ratio^3 fine cells, components 0..ncomp-1. */
int pcg_average_down(const pcg_array4* fine, pcg_array4* crse, const int32_t fine_lo[3], const int32_t fine_hi[3],
                     int32_t ratio, int32_t ncomp, pcg_stream_t stream);

/* ---- launch tuning ------------------------------------------------------------- */

/* Each heavy stage (0 ctoprim, 2 trace, 3-5 Riemann stages) exists in three register
 * budgets (variants 0-2, increasingly tight); the library keeps the variant used
 * per (precision_mode, nspec, stage). The trace of PCG_PREC_MIXED has variants 3-5 as
 * well: the same budgets for the tiled trace, which stages each tile of the FP32
 * primitive state and its halo in shared memory with one TMA load (plain PPM and PLM;
 * the hybrid-WENO trace is never tiled). particleclem_b200/autotune.py times them and
 * sets the fastest. No counterpart in the reference (AMReX chooses launch shapes). */
int pcg_set_launch_variant(int32_t precision_mode, int32_t nspec, int32_t stage, int32_t variant);
/* Current variant, or a negative PCG_E* code. */
int pcg_get_launch_variant(int32_t precision_mode, int32_t nspec, int32_t stage);

#ifdef __cplusplus
}
#endif
#endif
