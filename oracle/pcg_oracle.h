/*
 * pcg_oracle.h -- CPU FP64 oracle for PeleC's unsplit Godunov hydro advance.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker: a plain-C restatement of the
 * reference algorithm, used by tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg of bench.py. It is never linked into, called by, or a fallback for the product.
 *
 * Parity status: the hydro algorithm is pinned against the reference's own source
 * (Source/Godunov.cpp, PPM.cpp and the Godunov/PPM/PLM/Riemann/Hydro/PeleCUtilities
 * headers) compiled in place by oracle/ref/ against a minimal AMReX-API shim; see
 * oracle/ref/Makefile. The EOS (PelePhysics, not present in the reference checkout)
 * is a documented restatement shared by both, so absolute thermodynamic fidelity to
 * real PeleC is unpinned.
 *
 * Arrays use amrex::Array4 addressing: p[(i-b0) + (j-b1)*js + (k-b2)*ks + n*ns],
 * with end[] exclusive.
 */
#ifndef PCG_ORACLE_H
#define PCG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXNS 64

typedef struct {
  double* p;
  int64_t jstride, kstride, nstride;
  int32_t begin[3], end[3];
  int32_t ncomp;
} orc_array4;

typedef struct {
  double dx[3];
  double dt;
  double difmag;
  int32_t ppm_type, plm_iorder, use_flattening, use_hybrid_weno, weno_scheme;
  int32_t domlo[3], domhi[3], bclo[3], bchi[3];
  int32_t nspec;
  int32_t precision_mode;
} orc_params;

/* EOS set-up. kind 0: gamma law (nspec must be 1); kind 1: ideal-gas mixture with
 * NASA-7 polynomials. a_lo/a_hi hold 7 coefficients per species. */
int orc_set_eos_gamma(double gamma, double mw);
int orc_set_eos_nasa7(int nspec, const double* mw, const double* tmid,
                      const double* a_lo, const double* a_hi);

/* EOS point evaluations (exported for EOS parity tests). */
void orc_eos_rpy2cs(double r, double p, const double* y, double* cs);
void orc_eos_ryp2e(double r, const double* y, double p, double* e);
void orc_eos_rey2t(double r, double e, const double* y, double* t);
void orc_eos_rty2p(double r, double t, const double* y, double* p);
void orc_eos_rty2cs(double r, double t, const double* y, double* cs);
void orc_eos_rty2g(double r, double t, const double* y, double* g);
void orc_eos_rty2dpde_dpdre(double r, double t, const double* y, double* dpde, double* dpdr_e);
void orc_eos_y2wbar(const double* y, double* wbar);
void orc_eos_t2ei(double t, double* ei);
int orc_eos_nspec(void);

/* pc_ctoprim over box [lo,hi]: u -> q (QVAR), qaux (NQAUX). */
int orc_ctoprim(const int32_t lo[3], const int32_t hi[3], const orc_array4* u,
                orc_array4* q, orc_array4* qaux);

/* pc_umdrv for one box [lo,hi]. uout is accumulated into (caller zeroes it), flx[3]
 * is overwritten (area-weighted). srcq may be NULL (no sources: srcq == 0). */
int orc_umdrv(const orc_params* prm, const int32_t lo[3], const int32_t hi[3],
              const orc_array4* uin, orc_array4* uout, const orc_array4* q,
              const orc_array4* qaux, const orc_array4* srcq, orc_array4* flx,
              const orc_array4* area, const orc_array4* vol);

/* One construct_hydro_source box iteration: ctoprim on grow(bx,4), zero sources,
 * pc_umdrv. hydro_source (uout) is zeroed first, as Hydro.cpp:47 does. */
/* pc_srctoprim over [lo, hi] (Source/Hydro.H:14-68). */
int orc_srctoprim(const int32_t lo[3], const int32_t hi[3], const orc_array4* q, const orc_array4* qaux,
                  const orc_array4* src, orc_array4* srcq);
/* pc_umeth_3D alone (Source/Godunov.H:1142-1162): final fluxes, qec, pdivu. */
int orc_umeth(const orc_params* prm, const int32_t lo[3], const int32_t hi[3], const orc_array4* q,
              const orc_array4* qaux, const orc_array4* srcq, orc_array4* flx, orc_array4* qec,
              const orc_array4* area, orc_array4* pdivu, const orc_array4* vol);
int orc_hydro_box(const orc_params* prm, const int32_t lo[3], const int32_t hi[3],
                  const orc_array4* uin, orc_array4* uout, orc_array4* flx,
                  const orc_array4* area, const orc_array4* vol);

/* pc_estdt_hydro over [lo,hi] (the min over cells, before the cfl factor). */
double orc_estdt(const int32_t lo[3], const int32_t hi[3], const orc_array4* u,
                 const double dx[3]);

/* construct_Snew (S_new = S_old + dt * hydro_source) followed by computeTemp
 * (pc_rst_int_e default branch + pc_cmpTemp) over [lo,hi]. */
int orc_update_state(const int32_t lo[3], const int32_t hi[3], const orc_array4* s_old,
                     const orc_array4* hydro_source, double dt, orc_array4* s_new);

#ifdef __cplusplus
}
#endif
#endif
