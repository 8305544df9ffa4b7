/*
 * pcg_oracle.c -- CPU FP64 oracle (TEST INFRASTRUCTURE ONLY) for PeleC's unsplit
 * Godunov hydro advance. See pcg_oracle.h for the parity status.
 *
 * Every routine restates the reference routine it cites (paths relative to the
 * reference project root) with the same loops, box ranges and operation order, so
 * that a build without FMA contraction reproduces the reference bit for bit.
 * amrex::min/max follow std::min/std::max: min(a,b) = (b < a) ? b : a,
 * max(a,b) = (a < b) ? b : a.
 */
#include "pcg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- indices */
/* Source/IndexDefines.H:6-89 with NUM_ADV = NUM_AUX = NUM_LIN = 0. */
enum { URHO = 0, UMX = 1, UMY = 2, UMZ = 3, UEDEN = 4, UEINT = 5, UTEMP = 6, UFS = 7 };
enum { QRHO = 0, QU = 1, QV = 2, QW = 3, QGAME = 4, QPRES = 5, QREINT = 6, QTEMP = 7, QFS = 8 };
enum { QGAMC = 0, QC = 1, QCSML = 2, QDPDR = 3, QDPDE = 4, QRSPEC = 5, NQAUX = 6 };
enum { GDRHO = 0, GDU = 1, GDV = 2, GDW = 3, GDPRES = 4, GDGAME = 5, NGDNV = 6 };
/* Source/PeleC.H:49-57 (PCPhysBCType == amrex::PhysBCType numbering). */
enum { BC_INTERIOR = 0, BC_INFLOW, BC_OUTFLOW, BC_SYMMETRY, BC_SLIP_WALL, BC_NO_SLIP_WALL, BC_USER };

static int g_ns = 1; /* NUM_SPECIES of the current EOS */
#define NVAR (7 + g_ns)
#define QVAR (8 + g_ns)
#define MAXQ (8 + ORC_MAXNS)

/* Source/Constants.H:18-30 */
#define SMALLU 1.0e-12
#define SMALL_NUM 1.0e-8
#define VERY_SMALL_NUM (DBL_EPSILON * 1e-100)

static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static inline double dmax(double a, double b) { return (a < b) ? b : a; }

/* ---------------------------------------------------------------- boxes/fabs */
typedef struct { int lo[3], hi[3]; } box_t;
typedef struct {
  double* p;
  int lo[3], hi[3];
  int64_t js, ks, ns;
  int nc;
  int owned;
} fab_t;

static box_t mkbox(const int32_t lo[3], const int32_t hi[3]) {
  box_t b;
  for (int d = 0; d < 3; ++d) { b.lo[d] = lo[d]; b.hi[d] = hi[d]; }
  return b;
}
static box_t bgrow(box_t b, int n) {
  for (int d = 0; d < 3; ++d) { b.lo[d] -= n; b.hi[d] += n; }
  return b;
}
static box_t bgrow_dir(box_t b, int d, int n) { b.lo[d] -= n; b.hi[d] += n; return b; }
static box_t bgrow_hi(box_t b, int d, int n) { b.hi[d] += n; return b; }
static box_t bnodes(box_t b, int d) { b.hi[d] += 1; return b; } /* surroundingNodes */

static fab_t fab_new(box_t b, int nc) {
  fab_t f;
  for (int d = 0; d < 3; ++d) { f.lo[d] = b.lo[d]; f.hi[d] = b.hi[d]; }
  int64_t nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
  f.js = nx; f.ks = nx * ny; f.ns = nx * ny * nz; f.nc = nc;
  f.p = (double*)calloc((size_t)(f.ns * nc), sizeof(double));
  f.owned = 1;
  return f;
}
static void fab_free(fab_t* f) { if (f->owned) free(f->p); f->p = NULL; }
static fab_t fab_view(const orc_array4* a) {
  fab_t f;
  f.p = a->p;
  for (int d = 0; d < 3; ++d) { f.lo[d] = a->begin[d]; f.hi[d] = a->end[d] - 1; }
  f.js = a->jstride; f.ks = a->kstride; f.ns = a->nstride; f.nc = a->ncomp; f.owned = 0;
  return f;
}
#define F(f, i, j, k, n) \
  ((f).p[((i) - (f).lo[0]) + ((int64_t)(j) - (f).lo[1]) * (f).js + \
         ((int64_t)(k) - (f).lo[2]) * (f).ks + (int64_t)(n) * (f).ns])
static int fab_contains(const fab_t* f, int i, int j, int k) {
  return i >= f->lo[0] && i <= f->hi[0] && j >= f->lo[1] && j <= f->hi[1] &&
         k >= f->lo[2] && k <= f->hi[2];
}
#define FOR_BOX(b, i, j, k) \
  for (int k = (b).lo[2]; k <= (b).hi[2]; ++k) \
    for (int j = (b).lo[1]; j <= (b).hi[1]; ++j) \
      for (int i = (b).lo[0]; i <= (b).hi[0]; ++i)

/* ---------------------------------------------------------------- EOS */
/* PelePhysics' eos() is not part of the reference checkout. This is the documented
 * restatement used by every implementation in this project:
 *   rmix = RU * sum_k Y_k / W_k  (k ascending)
 *   gamma law: cs = sqrt(gamma*P/R), e = P/((gamma-1)*R), T = e*(gamma-1)/rmix,
 *              P = R*rmix*T, dp/de = (gamma-1)*R, dp/drho|e = rmix*T
 *   mixture:   cv_k, e_k from NASA-7 (range chosen by T < Tmid_k), cv = sum Y_k cv_k,
 *              e = sum Y_k e_k, T(R,P) = P/(R*rmix), G = (cv+rmix)/cv,
 *              cs = sqrt(G*P/R); T(e) by Newton from the stored T.  */
#define RU 8.31446261815324e7 /* erg / (mol K) */
#define NEWTON_MAXIT 20
#define NEWTON_RTOL 1.0e-10
#define NEWTON_TMIN 10.0

static struct {
  int kind; /* 0 gamma law, 1 NASA-7 mixture */
  double gamma;
  double imw[ORC_MAXNS];
  double tmid[ORC_MAXNS];
  double cvc[ORC_MAXNS][2][5];
  double ec[ORC_MAXNS][2][6];
} E;

int orc_set_eos_gamma(double gamma, double mw) {
  memset(&E, 0, sizeof(E));
  E.kind = 0;
  E.gamma = gamma;
  E.imw[0] = 1.0 / mw;
  g_ns = 1;
  return 0;
}

int orc_set_eos_nasa7(int nspec, const double* mw, const double* tmid, const double* a_lo,
                      const double* a_hi) {
  if (nspec < 1 || nspec > ORC_MAXNS) return -1;
  memset(&E, 0, sizeof(E));
  E.kind = 1;
  g_ns = nspec;
  for (int k = 0; k < nspec; ++k) {
    const double rw = RU / mw[k];
    E.imw[k] = 1.0 / mw[k];
    E.tmid[k] = tmid[k];
    for (int r = 0; r < 2; ++r) {
      const double* a = (r == 0 ? a_lo : a_hi) + 7 * k;
      E.cvc[k][r][0] = rw * (a[0] - 1.0);
      E.cvc[k][r][1] = rw * a[1];
      E.cvc[k][r][2] = rw * a[2];
      E.cvc[k][r][3] = rw * a[3];
      E.cvc[k][r][4] = rw * a[4];
      E.ec[k][r][0] = rw * a[5];
      E.ec[k][r][1] = rw * (a[0] - 1.0);
      E.ec[k][r][2] = rw * (a[1] / 2.0);
      E.ec[k][r][3] = rw * (a[2] / 3.0);
      E.ec[k][r][4] = rw * (a[3] / 4.0);
      E.ec[k][r][5] = rw * (a[4] / 5.0);
    }
  }
  return 0;
}

int orc_eos_nspec(void) { return g_ns; }

static double eos_rmix(const double* y) {
  double s = 0.0;
  for (int k = 0; k < g_ns; ++k) s = s + y[k] * E.imw[k];
  return RU * s;
}
static double mix_cv(double t, const double* y) {
  double cv = 0.0;
  for (int k = 0; k < g_ns; ++k) {
    const double* c = E.cvc[k][t < E.tmid[k] ? 0 : 1];
    const double cvk = c[0] + t * (c[1] + t * (c[2] + t * (c[3] + t * c[4])));
    cv = cv + y[k] * cvk;
  }
  return cv;
}
static double mix_e(double t, const double* y) {
  double e = 0.0;
  for (int k = 0; k < g_ns; ++k) {
    const double* c = E.ec[k][t < E.tmid[k] ? 0 : 1];
    const double ek = c[0] + t * (c[1] + t * (c[2] + t * (c[3] + t * (c[4] + t * c[5]))));
    e = e + y[k] * ek;
  }
  return e;
}

void orc_eos_rpy2cs(double r, double p, const double* y, double* cs) {
  if (E.kind == 0) { *cs = sqrt(E.gamma * p / r); return; }
  const double rmix = eos_rmix(y);
  const double t = p / (r * rmix);
  const double cv = mix_cv(t, y);
  const double g = (cv + rmix) / cv;
  *cs = sqrt(g * p / r);
}
void orc_eos_ryp2e(double r, const double* y, double p, double* e) {
  if (E.kind == 0) { *e = p / ((E.gamma - 1.0) * r); return; }
  const double rmix = eos_rmix(y);
  const double t = p / (r * rmix);
  *e = mix_e(t, y);
}
void orc_eos_rey2t(double r, double e, const double* y, double* t) {
  (void)r;
  const double rmix = eos_rmix(y);
  if (E.kind == 0) { *t = e * (E.gamma - 1.0) / rmix; return; }
  double tt = *t;
  if (!(tt > 0.0)) tt = 1000.0;
  for (int it = 0; it < NEWTON_MAXIT; ++it) {
    const double ek = mix_e(tt, y);
    const double cvk = mix_cv(tt, y);
    const double dt = (e - ek) / cvk;
    tt = tt + dt;
    if (tt < NEWTON_TMIN) tt = NEWTON_TMIN;
    if (fabs(dt) <= NEWTON_RTOL * tt) break;
  }
  *t = tt;
}
void orc_eos_rty2p(double r, double t, const double* y, double* p) {
  *p = r * eos_rmix(y) * t;
}
void orc_eos_rty2cs(double r, double t, const double* y, double* cs) {
  const double rmix = eos_rmix(y);
  const double p = r * rmix * t;
  if (E.kind == 0) { *cs = sqrt(E.gamma * p / r); return; }
  const double cv = mix_cv(t, y);
  const double g = (cv + rmix) / cv;
  *cs = sqrt(g * p / r);
}
void orc_eos_rty2g(double r, double t, const double* y, double* g) {
  (void)r;
  if (E.kind == 0) { *g = E.gamma; return; }
  const double cv = mix_cv(t, y);
  *g = (cv + eos_rmix(y)) / cv;
}
void orc_eos_rty2dpde_dpdre(double r, double t, const double* y, double* dpde, double* dpdr_e) {
  const double rmix = eos_rmix(y);
  if (E.kind == 0) {
    *dpde = (E.gamma - 1.0) * r;
  } else {
    *dpde = r * rmix / mix_cv(t, y);
  }
  *dpdr_e = rmix * t;
}
void orc_eos_y2wbar(const double* y, double* wbar) {
  double s = 0.0;
  for (int k = 0; k < g_ns; ++k) s = s + y[k] * E.imw[k];
  *wbar = 1.0 / s;
}

void orc_eos_t2ei(double t, double* ei) {
  for (int k = 0; k < g_ns; ++k) {
    if (E.kind == 0) {
      ei[k] = RU * E.imw[k] * t / (E.gamma - 1.0);
    } else {
      const double* c = E.ec[k][t < E.tmid[k] ? 0 : 1];
      ei[k] = c[0] + t * (c[1] + t * (c[2] + t * (c[3] + t * (c[4] + t * c[5]))));
    }
  }
}

/* ---------------------------------------------------------------- ctoprim */
/* Source/PeleCUtilities.H:242-320 (pc_ctoprim), omega = rad = 0. */
static void ctoprim_cell(int i, int j, int k, const fab_t* u, fab_t* q, fab_t* qa) {
  const double rho = F(*u, i, j, k, URHO);
  const double rhoinv = 1.0 / rho;
  const double vx = F(*u, i, j, k, UMX) * rhoinv;
  const double vy = F(*u, i, j, k, UMY) * rhoinv;
  const double vz = F(*u, i, j, k, UMZ) * rhoinv;
  const double kineng = 0.5 * rho * (vx * vx + vy * vy + vz * vz) - 0.5 * rho * 0.0 * 0.0 * 0.0 * 0.0;
  F(*q, i, j, k, QRHO) = rho;
  F(*q, i, j, k, QU) = vx;
  F(*q, i, j, k, QV) = vy;
  F(*q, i, j, k, QW) = vz;
  for (int n = 0; n < g_ns; n++) F(*q, i, j, k, QFS + n) = F(*u, i, j, k, UFS + n) / rho;
  const double e = (F(*u, i, j, k, UEDEN) - kineng) * rhoinv;
  double T = F(*u, i, j, k, UTEMP);
  double massfrac[ORC_MAXNS];
  for (int sp = 0; sp < g_ns; ++sp) {
    if ((-1e-4 * DBL_EPSILON < F(*q, i, j, k, sp + QFS)) &&
        (F(*q, i, j, k, sp + QFS) < 1e-4 * DBL_EPSILON)) {
      F(*q, i, j, k, sp + QFS) = 0.0;
    }
    massfrac[sp] = F(*q, i, j, k, sp + QFS);
  }
  double dpdr_e, dpde, gam1, cs, wbar, p;
  orc_eos_y2wbar(massfrac, &wbar);
  orc_eos_rey2t(rho, e, massfrac, &T);
  orc_eos_rty2p(rho, T, massfrac, &p);
  orc_eos_rty2cs(rho, T, massfrac, &cs);
  orc_eos_rty2g(rho, T, massfrac, &gam1);
  orc_eos_rty2dpde_dpdre(rho, T, massfrac, &dpde, &dpdr_e);
  F(*q, i, j, k, QTEMP) = T;
  F(*q, i, j, k, QREINT) = e * rho;
  F(*q, i, j, k, QPRES) = p;
  F(*q, i, j, k, QGAME) = p / (e * rho) + 1.0;
  F(*qa, i, j, k, QDPDR) = dpdr_e;
  F(*qa, i, j, k, QDPDE) = dpde;
  F(*qa, i, j, k, QGAMC) = gam1;
  F(*qa, i, j, k, QC) = cs;
  F(*qa, i, j, k, QCSML) = dmax(SMALL_NUM, SMALL_NUM * cs);
  F(*qa, i, j, k, QRSPEC) = RU / wbar;
}

int orc_ctoprim(const int32_t lo[3], const int32_t hi[3], const orc_array4* u, orc_array4* q,
                orc_array4* qaux) {
  fab_t uf = fab_view(u), qf = fab_view(q), af = fab_view(qaux);
  box_t b = mkbox(lo, hi);
  FOR_BOX(b, i, j, k) ctoprim_cell(i, j, k, &uf, &qf, &af);
  return 0;
}

/* Source/Hydro.H:14-68 (pc_srctoprim). */
static void srctoprim_cell(int i, int j, int k, const fab_t* q, const fab_t* qa, const fab_t* src,
                           fab_t* srcq) {
  const double srcrho = F(*src, i, j, k, URHO);
  const double rhoinv = 1.0 / F(*q, i, j, k, QRHO);
  const double vx = F(*q, i, j, k, QU);
  const double vy = F(*q, i, j, k, QV);
  const double vz = F(*q, i, j, k, QW);
  const double umx = F(*src, i, j, k, UMX);
  const double umy = F(*src, i, j, k, UMY);
  const double umz = F(*src, i, j, k, UMZ);
  F(*srcq, i, j, k, QRHO) = srcrho;
  F(*srcq, i, j, k, QU) = (umx - vx * srcrho) * rhoinv;
  F(*srcq, i, j, k, QV) = (umy - vy * srcrho) * rhoinv;
  F(*srcq, i, j, k, QW) = (umz - vz * srcrho) * rhoinv;
  F(*srcq, i, j, k, QREINT) = F(*src, i, j, k, UEDEN) - vx * umx - vy * umy - vz * umz +
                              srcrho * (vx * vx + vy * vy + vz * vz);
  F(*srcq, i, j, k, QPRES) =
    F(*qa, i, j, k, QDPDE) * (F(*srcq, i, j, k, QREINT) - F(*q, i, j, k, QREINT) * srcrho * rhoinv) *
      rhoinv +
    F(*qa, i, j, k, QDPDR) * srcrho;
  for (int n = 0; n < g_ns; n++)
    F(*srcq, i, j, k, QFS + n) = (F(*src, i, j, k, UFS + n) - F(*q, i, j, k, QFS + n) * srcrho) * rhoinv;
}

/* ---------------------------------------------------------------- flatten */
/* Source/Godunov.H:188-260 (flatten). q.contains() is tested against the q FAB. */
static double flatten(int i, int j, int k, int dir, const fab_t* q) {
  const int dv[3] = {dir == 0, dir == 1, dir == 2};
#define QS(s, n) F(*q, i + (s) * dv[0], j + (s) * dv[1], k + (s) * dv[2], n)
  if (!fab_contains(q, i + 3 * dv[0], j + 3 * dv[1], k + 3 * dv[2]) ||
      !fab_contains(q, i - 3 * dv[0], j - 3 * dv[1], k - 3 * dv[2]))
    return 1.0;
  const int n = QPRES;
  const double small_pres = 1.e-200;
  const double shktst = 0.33e0;
  const double zcut1 = 0.75e0;
  const double zcut2 = 0.85e0;
  const double dzcut = 1.0 / (zcut2 - zcut1);
  const double qm = QS(-1, n);
  const double qp = QS(1, n);
  const double qmun = QS(-1, QU + dir);
  const double qpun = QS(1, QU + dir);
  const double qmm = QS(-2, n);
  const double qpp = QS(2, n);
  double dp = qp - qm;
  const int ishft = (dp > 0.0) ? 1 : -1;
  double denom = dmax(small_pres, fabs(qpp - qmm));
  double zeta = fabs(dp) / denom;
  const double z = dmin(1.0, dmax(0.0, dzcut * (zeta - zcut1)));
  double tst = (qmun - qpun >= 0.0) ? 1.0 : 0.0;
  double tmp = dmin(qp, qm);
  const double chi = (fabs(dp) / tmp) > shktst ? tst : 0.0;
  const double qpshft = QS(1 - ishft, n);
  const double qmshft = QS(-(1 + ishft), n);
  const double qpunshft = QS(1 - ishft, QU + dir);
  const double qmunshft = QS(-(1 + ishft), QU + dir);
  const double qppshft = QS(2 - ishft, n);
  const double qmmshft = QS(-(2 + ishft), n);
  dp = qpshft - qmshft;
  denom = dmax(small_pres, fabs(qppshft - qmmshft));
  zeta = fabs(dp) / denom;
  const double z2 = dmin(1.0, dmax(0.0, dzcut * (zeta - zcut1)));
  tst = (qmunshft - qpunshft >= 0.0) ? 1.0 : 0.0;
  tmp = dmin(qpshft, qmshft);
  const double chi2 = (fabs(dp) / tmp) > shktst ? tst : 0.0;
  return 1.0 - dmax(chi2 * z2, chi * z);
#undef QS
}

/* ---------------------------------------------------------------- PPM */
/* Source/PPM.H:28-115 (ppm_reconstruct). s = {im2, im1, i0, ip1, ip2}. */
static void ppm_reconstruct(const double* s, double flatn, double* smo, double* spo) {
  double dsl = 2.0 * (s[1] - s[0]);
  double dsr = 2.0 * (s[2] - s[1]);
  double dsvl_l = 0.0;
  if (dsl * dsr > 0.0) {
    double dsc = 0.5 * (s[2] - s[0]);
    dsvl_l = copysign(1.0, dsc) * dmin(fabs(dsc), dmin(fabs(dsl), fabs(dsr)));
  }
  dsl = 2.0 * (s[2] - s[1]);
  dsr = 2.0 * (s[3] - s[2]);
  double dsvl_r = 0.0;
  if (dsl * dsr > 0.0) {
    double dsc = 0.5 * (s[3] - s[1]);
    dsvl_r = copysign(1.0, dsc) * dmin(fabs(dsc), dmin(fabs(dsl), fabs(dsr)));
  }
  double sm = 0.5 * (s[2] + s[1]) - (1.0 / 6.0) * (dsvl_r - dsvl_l);
  sm = dmax(sm, dmin(s[2], s[1]));
  sm = dmin(sm, dmax(s[2], s[1]));
  dsl = 2.0 * (s[2] - s[1]);
  dsr = 2.0 * (s[3] - s[2]);
  dsvl_l = 0.0;
  if (dsl * dsr > 0.0) {
    double dsc = 0.5 * (s[3] - s[1]);
    dsvl_l = copysign(1.0, dsc) * dmin(fabs(dsc), dmin(fabs(dsl), fabs(dsr)));
  }
  dsl = 2.0 * (s[3] - s[2]);
  dsr = 2.0 * (s[4] - s[3]);
  dsvl_r = 0.0;
  if (dsl * dsr > 0.0) {
    double dsc = 0.5 * (s[4] - s[2]);
    dsvl_r = copysign(1.0, dsc) * dmin(fabs(dsc), dmin(fabs(dsl), fabs(dsr)));
  }
  double sp = 0.5 * (s[3] + s[2]) - (1.0 / 6.0) * (dsvl_r - dsvl_l);
  sp = dmax(sp, dmin(s[3], s[2]));
  sp = dmin(sp, dmax(s[3], s[2]));
  sm = flatn * sm + (1.0 - flatn) * s[2];
  sp = flatn * sp + (1.0 - flatn) * s[2];
  if ((sp - s[2]) * (s[2] - sm) <= 0.0) {
    sp = s[2];
    sm = s[2];
  } else if (fabs(sp - s[2]) >= 2.0 * fabs(sm - s[2])) {
    sp = 3.0 * s[2] - 2.0 * sm;
  } else if (fabs(sm - s[2]) >= 2.0 * fabs(sp - s[2])) {
    sm = 3.0 * s[2] - 2.0 * sp;
  }
  *smo = sm;
  *spo = sp;
}

/* Source/PPM.H:131-189 (ppm_int_profile). */
static void ppm_int_profile(double sm, double sp, double sc, double u, double c, double dtdx,
                            double* Ip, double* Im) {
  double s6 = 6.0 * sc - 3.0 * (sm + sp);
  const double speeds[3] = {u - c, u, u + c};
  for (int w = 0; w < 3; ++w) {
    double speed = speeds[w];
    double sigma = fabs(speed) * dtdx;
    if (speed <= 0.0) {
      Ip[w] = sp;
      Im[w] = sm + 0.5 * sigma * (sp - sm + (1.0 - (2.0 / 3.0) * sigma) * s6);
    } else {
      Ip[w] = sp - 0.5 * sigma * (sp - sm - (1.0 - (2.0 / 3.0) * sigma) * s6);
      Im[w] = sm;
    }
  }
}

/* Source/WENO.H: the hybrid-WENO edge values of cell s[c] (sm on its low face, sp on its
 * high face) that replace the PPM parabola in trace_ppm when use_hybrid_weno is set
 * (Source/PPM.cpp:120-172). Published schemes: WENO-JS5 (Jiang & Shu 1996), WENO-Z5
 * (Borges et al. 2008), WENO-Z7 (Balsara & Shu 2000 stencils with Z weights), WENO-Z3;
 * every expression keeps the reference's order of operations (pow(x, 2) is x * x). */
static const double WENO_EPS = 1e-6;
static inline double sq(double x) { return x * x; }

/* smoothness of the three 3-point substencils of a 5-point stencil seen from the high
 * face, and mirrored from the low face */
static void w5_beta_hi(const double* s, double* b) {
  b[2] = (13.0 / 12.0) * sq(s[0] - 2.0 * s[1] + s[2]) + 0.25 * sq(s[0] - 4.0 * s[1] + 3.0 * s[2]);
  b[1] = (13.0 / 12.0) * sq(s[1] - 2.0 * s[2] + s[3]) + 0.25 * (s[1] - s[3]) * (s[1] - s[3]);
  b[0] = (13.0 / 12.0) * sq(s[2] - 2.0 * s[3] + s[4]) + 0.25 * sq(3.0 * s[2] - 4.0 * s[3] + s[4]);
}
static void w5_beta_lo(const double* s, double* b) {
  b[2] = (13.0 / 12.0) * sq(s[4] - 2.0 * s[3] + s[2]) + 0.25 * sq(s[4] - 4.0 * s[3] + 3.0 * s[2]);
  b[1] = (13.0 / 12.0) * sq(s[3] - 2.0 * s[2] + s[1]) + 0.25 * (s[3] - s[1]) * (s[3] - s[1]);
  b[0] = (13.0 / 12.0) * sq(s[2] - 2.0 * s[1] + s[0]) + 0.25 * sq(3.0 * s[2] - 4.0 * s[1] + s[0]);
}
/* nonlinear weights from the smoothness indicators, in place: JS 1/(eps+b)^2, Z 1+(tau/(eps+b))^2 */
static void w_weights(double* b, int n, double tau, int z) {
  for (int m = 0; m < n; ++m)
    b[m] = z ? 1.0 + (tau / (WENO_EPS + b[m])) * (tau / (WENO_EPS + b[m]))
             : 1.0 / ((WENO_EPS + b[m]) * (WENO_EPS + b[m]));
}
static double w5_blend(const double* b, const double* v) {
  const double a2 = b[2], a1 = 6.0 * b[1], a0 = 3.0 * b[0];
  const double ai = 1.0 / (a2 + a1 + a0);
  return (1.0 / 6.0) * ai * (a2 * v[2] + a1 * v[1] + a0 * v[0]);
}
static void weno5(const double* s, int z, double* sm, double* sp) {
  double b[3], v[3];
  w5_beta_hi(s, b);
  w_weights(b, 3, fabs(b[2] - b[0]), z);
  v[2] = 2.0 * s[0] - 7.0 * s[1] + 11.0 * s[2];
  v[1] = -s[1] + 5.0 * s[2] + 2.0 * s[3];
  v[0] = 2.0 * s[2] + 5.0 * s[3] - s[4];
  *sp = w5_blend(b, v);
  w5_beta_lo(s, b);
  w_weights(b, 3, fabs(b[2] - b[0]), z);
  v[2] = 11.0 * s[2] - 7.0 * s[3] + 2.0 * s[4];
  v[1] = -s[3] + 5.0 * s[2] + 2.0 * s[1];
  v[0] = 2.0 * s[2] + 5.0 * s[1] - s[0];
  *sm = w5_blend(b, v);
}
/* smoothness polynomial of the 4-point substencil (a, b, c, d) of WENO-7 with the
 * coefficient set k (the same shape for all four substencils) */
static double w7_beta(double a, double b, double c, double d, const double* k) {
  return a * (k[0] * a - k[1] * b + k[2] * c - k[3] * d) + b * (k[4] * b - k[5] * c + k[6] * d) +
         c * (k[7] * c - k[8] * d) + k[9] * (d * d);
}
static const double W7K[4][10] = {
  {2107.0, 9402.0, 7042.0, 1854.0, 11003.0, 17246.0, 4642.0, 7043.0, 3882.0, 547.0},
  {547.0, 2522.0, 1922.0, 494.0, 3443.0, 5966.0, 1602.0, 2843.0, 1642.0, 267.0},
  {267.0, 1642.0, 1602.0, 494.0, 2843.0, 5966.0, 1922.0, 3443.0, 2522.0, 547.0},
  {547.0, 3882.0, 4642.0, 1854.0, 7043.0, 17246.0, 7042.0, 11003.0, 9402.0, 2107.0},
};
static double w7_blend(const double* b, const double* v) {
  const double a3 = (1.0 / 35.0) * b[3], a2 = (12.0 / 35.0) * b[2], a1 = (18.0 / 35.0) * b[1],
               a0 = (4.0 / 35.0) * b[0];
  const double ai = 1.0 / (a3 + a2 + a1 + a0);
  return (1.0 / 12.0) * ai * (a3 * v[3] + a2 * v[2] + a1 * v[1] + a0 * v[0]);
}
static void weno7z(const double* s, double* sm, double* sp) {
  double b[4], v[4];
  b[3] = w7_beta(s[0], s[1], s[2], s[3], W7K[3]);
  b[2] = w7_beta(s[1], s[2], s[3], s[4], W7K[2]);
  b[1] = w7_beta(s[2], s[3], s[4], s[5], W7K[1]);
  b[0] = w7_beta(s[3], s[4], s[5], s[6], W7K[0]);
  w_weights(b, 4, fabs(b[3] - b[0]), 1);
  v[3] = -3.0 * s[0] + 13.0 * s[1] - 23.0 * s[2] + 25.0 * s[3];
  v[2] = s[1] - 5.0 * s[2] + 13.0 * s[3] + 3.0 * s[4];
  v[1] = -s[2] + 7.0 * s[3] + 7.0 * s[4] - s[5];
  v[0] = 3.0 * s[3] + 13.0 * s[4] - 5.0 * s[5] + s[6];
  *sp = w7_blend(b, v);
  b[3] = w7_beta(s[6], s[5], s[4], s[3], W7K[3]);
  b[2] = w7_beta(s[5], s[4], s[3], s[2], W7K[2]);
  b[1] = w7_beta(s[4], s[3], s[2], s[1], W7K[1]);
  b[0] = w7_beta(s[3], s[2], s[1], s[0], W7K[0]);
  w_weights(b, 4, fabs(b[3] - b[0]), 1);
  v[3] = -3.0 * s[6] + 13.0 * s[5] - 23.0 * s[4] + 25.0 * s[3];
  v[2] = s[5] - 5.0 * s[4] + 13.0 * s[3] + 3.0 * s[2];
  v[1] = -s[4] + 7.0 * s[3] + 7.0 * s[2] - s[1];
  v[0] = 3.0 * s[3] + 13.0 * s[2] - 5.0 * s[1] + s[0];
  *sm = w7_blend(b, v);
}
static void weno3z(const double* s, double* sm, double* sp) {
  double b[2];
  b[1] = (s[0] - s[1]) * (s[0] - s[1]);
  b[0] = (s[1] - s[2]) * (s[1] - s[2]);
  w_weights(b, 2, fabs(b[1] - b[0]), 1);
  double a1 = 2.0 * b[1], a0 = 1.0 * b[0], ai = 1.0 / (a1 + a0);
  *sp = 0.5 * ai * (a1 * (-s[0] + 3.0 * s[1]) + a0 * (s[1] + s[2]));
  b[1] = (s[2] - s[1]) * (s[2] - s[1]);
  b[0] = (s[1] - s[0]) * (s[1] - s[0]);
  w_weights(b, 2, fabs(b[1] - b[0]), 1);
  a1 = 2.0 * b[1];
  a0 = 1.0 * b[0];
  ai = 1.0 / (a1 + a0);
  *sm = 0.5 * ai * (a1 * (3.0 * s[1] - s[2]) + a0 * (s[0] + s[1]));
}

/* Source/PPM.cpp:6-424 (trace_ppm, ORIGINAL PPM branch; bx == vbx as called from
 * Godunov.cpp:188-200, so both face states are written for every cell). */
static void trace_ppm(box_t bx, int idir, const fab_t* q, fab_t* qm, fab_t* qp, double dt,
                      const double* dx, int use_flattening, int use_hybrid_weno, int weno_scheme) {
  const double dtdx = dt / dx[idir];
  const int QUN = (idir == 0) ? QU : (idir == 1) ? QV : QW;
  const int QUT = (idir == 0) ? QV : (idir == 1) ? QW : QU;
  const int QUTT = (idir == 0) ? QW : (idir == 1) ? QU : QV;
  const int dv[3] = {idir == 0, idir == 1, idir == 2};
  FOR_BOX(bx, i, j, k) {
    const int ip = i + dv[0], jp = j + dv[1], kp = k + dv[2];
    double massfrac[ORC_MAXNS];
    for (int s = 0; s < g_ns; ++s) massfrac[s] = F(*q, i, j, k, s + QFS);
    double cc = 0;
    orc_eos_rpy2cs(F(*q, i, j, k, QRHO), F(*q, i, j, k, QPRES), massfrac, &cc);
    double un = F(*q, i, j, k, QUN);
    double flat = 1.0;
    if (use_flattening) {
      for (int df = 0; df < 3; df++) flat = dmin(flat, flatten(i, j, k, df, q));
    }
    double Ip[MAXQ][3], Im[MAXQ][3];
    for (int n = 0; n < QVAR; n++) {
      double s[7], sm, sp;
      if (use_hybrid_weno && weno_scheme == 2) {
        /* on the outer ring of bx the stencil leaves q's grow(bx,4) box (the reference reads
         * beyond its allocation there); those traces feed no output, the read is clamped */
        for (int o = -3; o <= 3; ++o) {
          int c[3] = {i + o * dv[0], j + o * dv[1], k + o * dv[2]};
          for (int e = 0; e < 3; ++e) c[e] = c[e] < q->lo[e] ? q->lo[e] : c[e] > q->hi[e] ? q->hi[e] : c[e];
          s[o + 3] = F(*q, c[0], c[1], c[2], n);
        }
        weno7z(s, &sm, &sp);
        ppm_int_profile(sm, sp, s[3], un, cc, dtdx, Ip[n], Im[n]);
      } else if (use_hybrid_weno && weno_scheme == 3) {
        for (int o = -1; o <= 1; ++o) s[o + 1] = F(*q, i + o * dv[0], j + o * dv[1], k + o * dv[2], n);
        weno3z(s, &sm, &sp);
        ppm_int_profile(sm, sp, s[1], un, cc, dtdx, Ip[n], Im[n]);
      } else {
        for (int o = -2; o <= 2; ++o) s[o + 2] = F(*q, i + o * dv[0], j + o * dv[1], k + o * dv[2], n);
        if (use_hybrid_weno && (weno_scheme == 0 || weno_scheme == 1))
          weno5(s, weno_scheme == 1, &sm, &sp);
        else
          ppm_reconstruct(s, flat, &sm, &sp);
        ppm_int_profile(sm, sp, s[2], un, cc, dtdx, Ip[n], Im[n]);
      }
    }
    for (int n = QFS; n < g_ns + QFS; n++) {
      F(*qp, i, j, k, n) = Im[n][1];
      F(*qm, ip, jp, kp, n) = Ip[n][1];
    }
    /* plus state on face i */
    {
      double rho_ref = Im[QRHO][0];
      double un_ref = Im[QUN][0];
      double p_ref = Im[QPRES][0];
      double rhoe_g_ref = Im[QREINT][0];
      rho_ref = dmax(rho_ref, DBL_MIN);
      double rho_ref_inv = 1.0 / rho_ref;
      p_ref = dmax(p_ref, DBL_MIN);
      double massfrac_ref[ORC_MAXNS];
      for (int s = 0; s < g_ns; ++s) massfrac_ref[s] = Im[s + QFS][0];
      double cc_ref = 0;
      orc_eos_rpy2cs(rho_ref, p_ref, massfrac_ref, &cc_ref);
      double csq_ref = cc_ref * cc_ref;
      double cc_ref_inv = 1.0 / cc_ref;
      double h_g_ref = (p_ref + rhoe_g_ref) * rho_ref_inv;
      double dum = un_ref - Im[QUN][0];
      double dptotm = p_ref - Im[QPRES][0];
      double drho = rho_ref - Im[QRHO][1];
      double dptot = p_ref - Im[QPRES][1];
      double drhoe_g = rhoe_g_ref - Im[QREINT][1];
      double dup = un_ref - Im[QUN][2];
      double dptotp = p_ref - Im[QPRES][2];
      double alpham = 0.5 * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
      double alphap = 0.5 * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
      double alpha0r = drho - dptot / csq_ref;
      double alpha0e_g = drhoe_g - dptot * h_g_ref / csq_ref;
      (void)alpha0e_g;
      alpham = un - cc > 0.0 ? 0.0 : -alpham;
      alphap = un + cc > 0.0 ? 0.0 : -alphap;
      alpha0r = un > 0.0 ? 0.0 : -alpha0r;
      F(*qp, i, j, k, QRHO) = dmax(DBL_MIN, rho_ref + alphap + alpham + alpha0r);
      F(*qp, i, j, k, QUN) = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
      F(*qp, i, j, k, QPRES) = dmax(DBL_MIN, p_ref + (alphap + alpham) * csq_ref);
      F(*qp, i, j, k, QUT) = Im[QUT][1];
      F(*qp, i, j, k, QUTT) = Im[QUTT][1];
      double eint = 0;
      double massfrac_p[ORC_MAXNS];
      for (int s = 0; s < g_ns; ++s) massfrac_p[s] = F(*qp, i, j, k, s + QFS);
      orc_eos_ryp2e(F(*qp, i, j, k, QRHO), massfrac_p, F(*qp, i, j, k, QPRES), &eint);
      F(*qp, i, j, k, QREINT) = F(*qp, i, j, k, QRHO) * eint;
    }
    /* minus state on face i+1 */
    {
      double rho_ref = Ip[QRHO][2];
      double un_ref = Ip[QUN][2];
      double p_ref = Ip[QPRES][2];
      double rhoe_g_ref = Ip[QREINT][2];
      rho_ref = dmax(rho_ref, DBL_MIN);
      double rho_ref_inv = 1.0 / rho_ref;
      p_ref = dmax(p_ref, DBL_MIN);
      double massfrac_ref[ORC_MAXNS];
      for (int s = 0; s < g_ns; ++s) massfrac_ref[s] = Ip[s + QFS][2];
      double cc_ref = 0;
      orc_eos_rpy2cs(rho_ref, p_ref, massfrac_ref, &cc_ref);
      double csq_ref = cc_ref * cc_ref;
      double cc_ref_inv = 1.0 / cc_ref;
      double h_g_ref = (p_ref + rhoe_g_ref) * rho_ref_inv;
      double dum = un_ref - Ip[QUN][0];
      double dptotm = p_ref - Ip[QPRES][0];
      double drho = rho_ref - Ip[QRHO][1];
      double dptot = p_ref - Ip[QPRES][1];
      double drhoe_g = rhoe_g_ref - Ip[QREINT][1];
      double dup = un_ref - Ip[QUN][2];
      double dptotp = p_ref - Ip[QPRES][2];
      double alpham = 0.5 * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
      double alphap = 0.5 * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
      double alpha0r = drho - dptot / csq_ref;
      double alpha0e_g = drhoe_g - dptot * h_g_ref / csq_ref;
      (void)alpha0e_g;
      alpham = un - cc > 0.0 ? -alpham : 0.0;
      alphap = un + cc > 0.0 ? -alphap : 0.0;
      alpha0r = un > 0.0 ? -alpha0r : 0.0;
      F(*qm, ip, jp, kp, QRHO) = dmax(DBL_MIN, rho_ref + alphap + alpham + alpha0r);
      F(*qm, ip, jp, kp, QUN) = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
      F(*qm, ip, jp, kp, QPRES) = dmax(DBL_MIN, p_ref + (alphap + alpham) * csq_ref);
      F(*qm, ip, jp, kp, QUT) = Ip[QUT][1];
      F(*qm, ip, jp, kp, QUTT) = Ip[QUTT][1];
      double eint = 0;
      double massfrac_m[ORC_MAXNS];
      for (int s = 0; s < g_ns; ++s) massfrac_m[s] = F(*qm, ip, jp, kp, s + QFS);
      orc_eos_ryp2e(F(*qm, ip, jp, kp, QRHO), massfrac_m, F(*qm, ip, jp, kp, QPRES), &eint);
      F(*qm, ip, jp, kp, QREINT) = F(*qm, ip, jp, kp, QRHO) * eint;
    }
  }
}

/* ---------------------------------------------------------------- PLM */
/* Source/PLM.H:21-77 (plm_slope). */
static double plm_slope(int i, int j, int k, int n, int dir, const fab_t* q, double flat, int order) {
  if (order == 1) return 0.0;
  const int dv[3] = {dir == 0, dir == 1, dir == 2};
  double dlft, drgt, dcen, dfm = 0.0, dfp = 0.0, dlim, dsgn, dtemp;
  const double qc = F(*q, i, j, k, n);
  const double qm2 = F(*q, i - 2 * dv[0], j - 2 * dv[1], k - 2 * dv[2], n);
  const double qm = F(*q, i - dv[0], j - dv[1], k - dv[2], n);
  const double qp = F(*q, i + dv[0], j + dv[1], k + dv[2], n);
  const double qp2 = F(*q, i + 2 * dv[0], j + 2 * dv[1], k + 2 * dv[2], n);
  if (order == 4) {
    dlft = qm - qm2;
    drgt = qc - qm;
    dcen = 0.5 * (dlft + drgt);
    dsgn = copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(fabs(dlft), fabs(drgt)) : 0.0;
    dfm = dsgn * dmin(dlim, fabs(dcen));
    dlft = qp - qc;
    drgt = qp2 - qp;
    dcen = 0.5 * (dlft + drgt);
    dsgn = copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(fabs(dlft), fabs(drgt)) : 0.0;
    dfp = dsgn * dmin(dlim, fabs(dcen));
  }
  dlft = qc - qm;
  drgt = qp - qc;
  dcen = 0.5 * (dlft + drgt);
  dsgn = copysign(1.0, dcen);
  dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(fabs(dlft), fabs(drgt)) : 0.0;
  dtemp = (order == 2) ? dcen : 4.0 / 3.0 * dcen - 1.0 / 6.0 * (dfp + dfm);
  return flat * dsgn * dmin(dlim, fabs(dtemp));
}

/* Source/PLM.H:167-309 (pc_plm_d). */
static void pc_plm_d(int i, int j, int k, int dir, fab_t* qm, fab_t* qp, const double* slope,
                     const fab_t* q, double cc, double dx, double dt) {
  const int dv[3] = {dir == 0, dir == 1, dir == 2};
  const int ip = i + dv[0], jp = j + dv[1], kp = k + dv[2];
  const int l1 = (dir == 0) ? 1 : 0;
  const int l2 = (dir == 2) ? 1 : 2;
  const double dtdx = dt / dx;
  const double cs = cc * cc;
  const double rho = F(*q, i, j, k, QRHO);
  const double vel[3] = {F(*q, i, j, k, QU), F(*q, i, j, k, QV), F(*q, i, j, k, QW)};
  const double p = F(*q, i, j, k, QPRES);
  const double rhoe = F(*q, i, j, k, QREINT);
  const double enth = ((rhoe + p) / rho) / cs;
  const double drho = slope[QRHO];
  const double dvel[3] = {slope[QU], slope[QV], slope[QW]};
  const double dp = slope[QPRES];
  const double drhoe = slope[QREINT];
  const double alpham = 0.5 * (dp / (rho * cc) - dvel[dir]) * rho / cc;
  const double alphap = 0.5 * (dp / (rho * cc) + dvel[dir]) * rho / cc;
  const double alpha0r = drho - dp / cs;
  const double alpha0e = drhoe - dp * enth;
  const double alpha0v = dvel[l1];
  const double alpha0w = dvel[l2];
  const double wv[3] = {vel[dir] - cc, vel[dir], vel[dir] + cc};

  double rho_ref = rho - 0.5 * (1.0 + dtdx * dmin(wv[0], 0.0)) * drho;
  double vel_ref[3];
  for (int dim = 0; dim < 3; dim++)
    vel_ref[dim] = vel[dim] - 0.5 * (1.0 + dtdx * dmin(wv[0], 0.0)) * dvel[dim];
  double p_ref = p - 0.5 * (1.0 + dtdx * dmin(wv[0], 0.0)) * dp;
  double rhoe_ref = rhoe - 0.5 * (1.0 + dtdx * dmin(wv[0], 0.0)) * drhoe;
  const double apright = 0.25 * dtdx * (wv[0] - wv[2]) * (1.0 - copysign(1.0, wv[2])) * alphap;
  const double amright = 0.0;
  const double azrright = 0.25 * dtdx * (wv[0] - wv[1]) * (1.0 - copysign(1.0, wv[1])) * alpha0r;
  const double azeright = 0.25 * dtdx * (wv[0] - wv[1]) * (1.0 - copysign(1.0, wv[1])) * alpha0e;
  const double azv1rght = 0.25 * dtdx * (wv[0] - wv[1]) * (1.0 - copysign(1.0, wv[1])) * alpha0v;
  const double azw1rght = 0.25 * dtdx * (wv[0] - wv[1]) * (1.0 - copysign(1.0, wv[1])) * alpha0w;
  F(*qp, i, j, k, QRHO) = rho_ref + apright + amright + azrright;
  F(*qp, i, j, k, QRHO) = dmax(DBL_MIN, F(*qp, i, j, k, QRHO));
  F(*qp, i, j, k, QU + dir) = vel_ref[dir] + (apright - amright) * cc / rho;
  F(*qp, i, j, k, QU + l1) = vel_ref[l1] + azv1rght;
  F(*qp, i, j, k, QU + l2) = vel_ref[l2] + azw1rght;
  F(*qp, i, j, k, QPRES) = p_ref + (apright + amright) * cs;
  F(*qp, i, j, k, QPRES) = dmax(F(*qp, i, j, k, QPRES), DBL_MIN);
  F(*qp, i, j, k, QREINT) = rhoe_ref + (apright + amright) * enth * cs + azeright;

  rho_ref = rho + 0.5 * (1.0 - dtdx * dmax(wv[2], 0.0)) * drho;
  for (int dim = 0; dim < 3; dim++)
    vel_ref[dim] = vel[dim] + 0.5 * (1.0 - dtdx * dmax(wv[2], 0.0)) * dvel[dim];
  p_ref = p + 0.5 * (1.0 - dtdx * dmax(wv[2], 0.0)) * dp;
  rhoe_ref = rhoe + 0.5 * (1.0 - dtdx * dmax(wv[2], 0.0)) * drhoe;
  const double apleft = 0.0;
  const double amleft = 0.25 * dtdx * (wv[2] - wv[0]) * (1.0 + copysign(1.0, wv[0])) * alpham;
  const double azrleft = 0.25 * dtdx * (wv[2] - wv[1]) * (1.0 + copysign(1.0, wv[1])) * alpha0r;
  const double azeleft = 0.25 * dtdx * (wv[2] - wv[1]) * (1.0 + copysign(1.0, wv[1])) * alpha0e;
  const double azv1left = 0.25 * dtdx * (wv[2] - wv[1]) * (1.0 + copysign(1.0, wv[1])) * alpha0v;
  const double azw1left = 0.25 * dtdx * (wv[2] - wv[1]) * (1.0 + copysign(1.0, wv[1])) * alpha0w;
  F(*qm, ip, jp, kp, QRHO) = rho_ref + apleft + amleft + azrleft;
  F(*qm, ip, jp, kp, QRHO) = dmax(F(*qm, ip, jp, kp, QRHO), DBL_MIN);
  F(*qm, ip, jp, kp, QU + dir) = vel_ref[dir] + (apleft - amleft) * cc / rho;
  F(*qm, ip, jp, kp, QU + l1) = vel_ref[l1] + azv1left;
  F(*qm, ip, jp, kp, QU + l2) = vel_ref[l2] + azw1left;
  F(*qm, ip, jp, kp, QPRES) = p_ref + (apleft + amleft) * cs;
  F(*qm, ip, jp, kp, QPRES) = dmax(F(*qm, ip, jp, kp, QPRES), DBL_MIN);
  F(*qm, ip, jp, kp, QREINT) = rhoe_ref + (apleft + amleft) * enth * cs + azeleft;

  const double vel_ad = F(*q, i, j, k, QU + dir);
  const double spzerom = (vel_ad > 0) ? -1.0 : vel_ad * dtdx;
  const double spzerop = (vel_ad >= 0) ? vel_ad * dtdx : 1.0;
  for (int n = 0; n < g_ns; n++) {
    const int c = QFS + n;
    const double acmprght = 0.5 * (-1.0 - spzerom) * slope[c];
    F(*qp, i, j, k, c) = F(*q, i, j, k, c) + acmprght;
    const double acmpleft = 0.5 * (1.0 - spzerop) * slope[c];
    F(*qm, ip, jp, kp, c) = F(*q, i, j, k, c) + acmpleft;
  }
}

/* ---------------------------------------------------------------- Riemann */
/* Source/Riemann.H:9-200 (riemann), omega = rad = 0. */
static void riemann(double rl, double ul, double vl, double v2l, double pl, const double* spl,
                    double rr, double ur, double vr, double v2r, double pr, const double* spr,
                    int bc_test_val, double cav, double* ustar_o, double* uflx_rho, double* uflx_u,
                    double* uflx_v, double* uflx_w, double* uflx_eden, double* uflx_eint,
                    double* qint_iu_o, double* qint_iv1_o, double* qint_iv2_o, double* qint_gdpres_o,
                    double* qint_gdgame_o) {
  const double wsmall = DBL_MIN;
  double gdnv_state_massfrac[ORC_MAXNS];
  for (int n = 0; n < g_ns; n++) gdnv_state_massfrac[n] = spl[n];
  double cl = 0.0;
  orc_eos_rpy2cs(rl, pl, gdnv_state_massfrac, &cl);
  for (int n = 0; n < g_ns; n++) gdnv_state_massfrac[n] = spr[n];
  double cr = 0.0;
  orc_eos_rpy2cs(rr, pr, gdnv_state_massfrac, &cr);
  const double wl = dmax(wsmall, cl * rl);
  const double wr = dmax(wsmall, cr * rr);
  const double pstar = dmax(DBL_MIN, ((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr));
  double ustar = ((wl * ul + wr * ur) + (pl - pr)) / (wl + wr);

  int mask = ustar > 0.0;
  double ro = 0.0;
  double rspo[ORC_MAXNS];
  for (int n = 0; n < g_ns; n++) {
    rspo[n] = mask ? rl * spl[n] : rr * spr[n];
    ro += rspo[n];
  }
  double uo = mask ? ul : ur;
  double po = mask ? pl : pr;
  mask = fabs(ustar) < SMALLU * 0.5 * (fabs(ul) + fabs(ur)) || ustar == 0.0;
  ustar = mask ? 0.0 : ustar;
  ro = 0.0;
  for (int n = 0; n < g_ns; n++) {
    rspo[n] = mask ? 0.5 * (rl * spl[n] + rr * spr[n]) : rspo[n];
    ro += rspo[n];
  }
  uo = mask ? 0.5 * (ul + ur) : uo;
  po = mask ? 0.5 * (pl + pr) : po;

  double gdnv_state_rho = ro;
  double gdnv_state_p = po;
  for (int n = 0; n < g_ns; n++) gdnv_state_massfrac[n] = rspo[n] / ro;
  double gdnv_state_e;
  orc_eos_ryp2e(gdnv_state_rho, gdnv_state_massfrac, gdnv_state_p, &gdnv_state_e);
  double co;
  orc_eos_rpy2cs(gdnv_state_rho, gdnv_state_p, gdnv_state_massfrac, &co);

  const double drho = (pstar - po) / (co * co);
  double rstar = 0.0;
  double rspstar[ORC_MAXNS];
  for (int n = 0; n < g_ns; n++) {
    const double spon = rspo[n] / ro;
    rspstar[n] = dmax(0.0, rspo[n] + drho * spon);
    rstar += rspstar[n];
  }
  gdnv_state_rho = rstar;
  gdnv_state_p = pstar;
  for (int n = 0; n < g_ns; n++) gdnv_state_massfrac[n] = rspstar[n] / rstar;
  orc_eos_ryp2e(gdnv_state_rho, gdnv_state_massfrac, gdnv_state_p, &gdnv_state_e);
  double cstar;
  orc_eos_rpy2cs(gdnv_state_rho, gdnv_state_p, gdnv_state_massfrac, &cstar);

  const double sgnm = copysign(1.0, ustar);
  double spout = co - sgnm * uo;
  double spin = cstar - sgnm * ustar;
  const double ushock = 0.5 * (spin + spout);
  mask = pstar < po;
  spout = mask ? spout : ushock;
  spin = mask ? spin : ushock;
  const double scr = (fabs(spout - spin) < VERY_SMALL_NUM) ? SMALL_NUM * cav : spout - spin;
  const double frac = dmax(0.0, dmin(1.0, (1.0 + (spout + spin) / scr) * 0.5));

  mask = ustar > 0.0;
  double qint_iv1 = mask ? vl : vr;
  double qint_iv2 = mask ? v2l : v2r;
  mask = (ustar == 0.0);
  qint_iv1 = mask ? 0.5 * (vl + vr) : qint_iv1;
  qint_iv2 = mask ? 0.5 * (v2l + v2r) : qint_iv2;
  double rgd = 0.0;
  double rspgd[ORC_MAXNS];
  for (int n = 0; n < g_ns; n++) {
    rspgd[n] = frac * rspstar[n] + (1.0 - frac) * rspo[n];
    rgd += rspgd[n];
  }
  double qint_iu = frac * ustar + (1.0 - frac) * uo;
  double qint_gdpres = frac * pstar + (1.0 - frac) * po;
  gdnv_state_rho = rgd;
  gdnv_state_p = qint_gdpres;
  for (int n = 0; n < g_ns; n++) gdnv_state_massfrac[n] = rspgd[n] / rgd;
  orc_eos_ryp2e(gdnv_state_rho, gdnv_state_massfrac, gdnv_state_p, &gdnv_state_e);

  mask = (spout < 0.0);
  rgd = 0.0;
  for (int n = 0; n < g_ns; n++) {
    rspgd[n] = mask ? rspo[n] : rspgd[n];
    rgd += rspgd[n];
  }
  qint_iu = mask ? uo : qint_iu;
  qint_gdpres = mask ? po : qint_gdpres;
  mask = (spin >= 0.0);
  rgd = 0.0;
  for (int n = 0; n < g_ns; n++) {
    rspgd[n] = mask ? rspstar[n] : rspgd[n];
    rgd += rspgd[n];
  }
  qint_iu = mask ? ustar : qint_iu;
  qint_gdpres = mask ? pstar : qint_gdpres;

  gdnv_state_rho = rgd;
  gdnv_state_p = qint_gdpres;
  for (int n = 0; n < g_ns; n++) gdnv_state_massfrac[n] = rspgd[n] / rgd;
  orc_eos_ryp2e(gdnv_state_rho, gdnv_state_massfrac, gdnv_state_p, &gdnv_state_e);
  double regd = gdnv_state_rho * gdnv_state_e;

  double qint_gdgame = qint_gdpres / regd + 1.0;
  qint_iu = bc_test_val * qint_iu;
  const double frho = rgd * qint_iu;
  *uflx_rho = frho;
  *uflx_u = frho * qint_iu + qint_gdpres;
  *uflx_v = frho * qint_iv1;
  *uflx_w = frho * qint_iv2;
  const double rhoetot = regd + 0.5 * rgd * (qint_iu * qint_iu + qint_iv1 * qint_iv1 + qint_iv2 * qint_iv2) -
                         0.5 * rgd * 0.0 * 0.0 * 0.0 * 0.0;
  *uflx_eden = qint_iu * (rhoetot + qint_gdpres);
  *uflx_eint = qint_iu * regd;
  *ustar_o = ustar;
  *qint_iu_o = qint_iu;
  *qint_iv1_o = qint_iv1;
  *qint_iv2_o = qint_iv2;
  *qint_gdpres_o = qint_gdpres;
  *qint_gdgame_o = qint_gdgame;
}

/* Source/Godunov.H:303-449 (pc_cmpflx) with pc_cmpflx_passive (:15-25). */
static void cmpflx(int i, int j, int k, int bclo, int bchi, int domlo, int domhi, const fab_t* ql,
                   const fab_t* qr, fab_t* flx, fab_t* qint, const fab_t* qa, int dir) {
  int IU, IV, IV2, GU, GV, GV2, f0, f1, f2;
  double cav;
  if (dir == 0) {
    IU = QU; IV = QV; IV2 = QW; GU = GDU; GV = GDV; GV2 = GDW;
    cav = 0.5 * (F(*qa, i, j, k, QC) + F(*qa, i - 1, j, k, QC));
    f0 = UMX; f1 = UMY; f2 = UMZ;
  } else if (dir == 1) {
    IU = QV; IV = QU; IV2 = QW; GU = GDV; GV = GDU; GV2 = GDW;
    cav = 0.5 * (F(*qa, i, j, k, QC) + F(*qa, i, j - 1, k, QC));
    f0 = UMY; f1 = UMX; f2 = UMZ;
  } else {
    IU = QW; IV = QU; IV2 = QV; GU = GDW; GV = GDU; GV2 = GDV;
    cav = 0.5 * (F(*qa, i, j, k, QC) + F(*qa, i, j, k - 1, QC));
    f0 = UMZ; f1 = UMX; f2 = UMY;
  }
  double spl[ORC_MAXNS], spr[ORC_MAXNS];
  for (int sp = 0; sp < g_ns; ++sp) {
    spl[sp] = F(*ql, i, j, k, QFS + sp);
    spr[sp] = F(*qr, i, j, k, QFS + sp);
  }
  double ul = F(*ql, i, j, k, IU), vl = F(*ql, i, j, k, IV), v2l = F(*ql, i, j, k, IV2);
  double pl = F(*ql, i, j, k, QPRES), rhol = F(*ql, i, j, k, QRHO);
  double ur = F(*qr, i, j, k, IU), vr = F(*qr, i, j, k, IV), v2r = F(*qr, i, j, k, IV2);
  double pr = F(*qr, i, j, k, QPRES), rhor = F(*qr, i, j, k, QRHO);
  const int idx = (dir == 2) ? k : ((dir == 0) ? i : j);
  if (idx == domlo) {
    if (bclo == BC_NO_SLIP_WALL || bclo == BC_SLIP_WALL || bclo == BC_SYMMETRY) {
      ul = -ur; vl = vr; v2l = v2r; pl = pr; rhol = rhor;
    } else if (bclo == BC_OUTFLOW) {
      ul = ur; vl = vr; v2l = v2r; pl = pr; rhol = rhor;
    }
  } else if (idx == domhi + 1) {
    if (bchi == BC_NO_SLIP_WALL || bchi == BC_SLIP_WALL || bchi == BC_SYMMETRY) {
      ur = -ul; vr = vl; v2r = v2l; pr = pl; rhor = rhol;
    } else if (bchi == BC_OUTFLOW) {
      ur = ul; vr = vl; v2r = v2l; pr = pl; rhor = rhol;
    }
  }
  double ustar, frho, fu, fv, fw, fe, fei, giu, giv1, giv2, gp, gg;
  riemann(rhol, ul, vl, v2l, pl, spl, rhor, ur, vr, v2r, pr, spr, 1, cav, &ustar, &frho, &fu, &fv,
          &fw, &fe, &fei, &giu, &giv1, &giv2, &gp, &gg);
  F(*flx, i, j, k, URHO) = frho;
  F(*flx, i, j, k, f0) = fu;
  F(*flx, i, j, k, f1) = fv;
  F(*flx, i, j, k, f2) = fw;
  F(*flx, i, j, k, UEDEN) = fe;
  F(*flx, i, j, k, UEINT) = fei;
  F(*qint, i, j, k, GU) = giu;
  F(*qint, i, j, k, GV) = giv1;
  F(*qint, i, j, k, GV2) = giv2;
  F(*qint, i, j, k, GDPRES) = gp;
  F(*qint, i, j, k, GDGAME) = gg;
  const double flxrho = frho;
  for (int n = 0; n < g_ns; n++) {
    const int qc = QFS + n;
    const double a = F(*ql, i, j, k, qc), b = F(*qr, i, j, k, qc);
    F(*flx, i, j, k, UFS + n) = (ustar > 0.0) ? flxrho * a : (ustar < 0.0) ? flxrho * b : flxrho * 0.5 * (a + b);
  }
}

/* ---------------------------------------------------------------- transverse */
/* Source/Godunov.H:455-633 (pc_transdo, regular geometry) with pc_transdo_passive (:30-73). */
static void transdo(int i, int j, int k, int dir, int other_dir, fab_t* qm, fab_t* qp,
                    const fab_t* qnormm, const fab_t* qnormp, const fab_t* flxx, const fab_t* qa,
                    const fab_t* qint, double cdtdx) {
  const int n1 = i + (dir == 0), n2 = j + (dir == 1), n3 = k + (dir == 2);
  const int t1 = i + (other_dir == 0), t2 = j + (other_dir == 1), t3 = k + (other_dir == 2);
  const int qvidx = (other_dir == 0) ? GDU : ((other_dir == 1) ? GDV : GDW);
  const double flxrho = cdtdx * (F(*flxx, t1, t2, t3, URHO) - F(*flxx, i, j, k, URHO));
  const double flxu = cdtdx * (F(*flxx, t1, t2, t3, UMX) - F(*flxx, i, j, k, UMX));
  const double flxv = cdtdx * (F(*flxx, t1, t2, t3, UMY) - F(*flxx, i, j, k, UMY));
  const double flxw = cdtdx * (F(*flxx, t1, t2, t3, UMZ) - F(*flxx, i, j, k, UMZ));
  const double flxe = cdtdx * (F(*flxx, t1, t2, t3, UEDEN) - F(*flxx, i, j, k, UEDEN));
  const double c = F(*qa, i, j, k, QGAMC);
  for (int n = 0; n < g_ns; n++) {
    const int uc = UFS + n, qc = QFS + n;
    const double compn = cdtdx * (F(*flxx, t1, t2, t3, uc) - F(*flxx, i, j, k, uc));
    double rr = F(*qnormp, i, j, k, QRHO);
    double rrnew = rr - flxrho;
    double compo = rr * F(*qnormp, i, j, k, qc) - compn;
    F(*qp, i, j, k, qc) = compo / rrnew;
    rr = F(*qnormm, n1, n2, n3, QRHO);
    rrnew = rr - flxrho;
    compo = rr * F(*qnormm, n1, n2, n3, qc) - compn;
    F(*qm, n1, n2, n3, qc) = compo / rrnew;
  }
  const double pggp = F(*qint, t1, t2, t3, GDPRES);
  const double pggm = F(*qint, i, j, k, GDPRES);
  const double ugp = F(*qint, t1, t2, t3, qvidx);
  const double ugm = F(*qint, i, j, k, qvidx);
  const double dAup = pggp * ugp - pggm * ugm;
  const double pav = 0.5 * (pggp + pggm);
  const double dAu = ugp - ugm;
  {
    const double rrr = F(*qnormp, i, j, k, QRHO);
    double rur = F(*qnormp, i, j, k, QU);
    double rvr = F(*qnormp, i, j, k, QV);
    double rwr = F(*qnormp, i, j, k, QW);
    const double ekinr = 0.5 * rrr * (rur * rur + rvr * rvr + rwr * rwr);
    rur *= rrr;
    rvr *= rrr;
    rwr *= rrr;
    const double rer = F(*qnormp, i, j, k, QREINT) + ekinr;
    const double rrnewr = rrr - flxrho;
    const double runewr = rur - flxu;
    const double rvnewr = rvr - flxv;
    const double rwnewr = rwr - flxw;
    const double renewr = rer - flxe;
    F(*qp, i, j, k, QRHO) = rrnewr;
    F(*qp, i, j, k, QU) = runewr / rrnewr;
    F(*qp, i, j, k, QV) = rvnewr / rrnewr;
    F(*qp, i, j, k, QW) = rwnewr / rrnewr;
    const double rhoekinr = 0.5 * (runewr * runewr + rvnewr * rvnewr + rwnewr * rwnewr) / rrnewr;
    F(*qp, i, j, k, QREINT) = renewr - rhoekinr;
    const double pnewr = F(*qnormp, i, j, k, QPRES) - cdtdx * (dAup + pav * dAu * (c - 1.0));
    F(*qp, i, j, k, QPRES) = dmax(pnewr, VERY_SMALL_NUM);
  }
  {
    const double rrl = F(*qnormm, n1, n2, n3, QRHO);
    double rul = F(*qnormm, n1, n2, n3, QU);
    double rvl = F(*qnormm, n1, n2, n3, QV);
    double rwl = F(*qnormm, n1, n2, n3, QW);
    const double ekinl = 0.5 * rrl * (rul * rul + rvl * rvl + rwl * rwl);
    rul *= rrl;
    rvl *= rrl;
    rwl *= rrl;
    const double rel = F(*qnormm, n1, n2, n3, QREINT) + ekinl;
    const double rrnewl = rrl - flxrho;
    const double runewl = rul - flxu;
    const double rvnewl = rvl - flxv;
    const double rwnewl = rwl - flxw;
    const double renewl = rel - flxe;
    F(*qm, n1, n2, n3, QRHO) = rrnewl;
    F(*qm, n1, n2, n3, QU) = runewl / rrnewl;
    F(*qm, n1, n2, n3, QV) = rvnewl / rrnewl;
    F(*qm, n1, n2, n3, QW) = rwnewl / rrnewl;
    const double rhoekinl = 0.5 * (runewl * runewl + rvnewl * rvnewl + rwnewl * rwnewl) / rrnewl;
    F(*qm, n1, n2, n3, QREINT) = renewl - rhoekinl;
    const double pnewl = F(*qnormm, n1, n2, n3, QPRES) - cdtdx * (dAup + pav * dAu * (c - 1.0));
    F(*qm, n1, n2, n3, QPRES) = dmax(pnewl, VERY_SMALL_NUM);
  }
}

/* Source/Godunov.H:639-845 (pc_transdd, regular geometry) with pc_transdd_passive (:78-132). */
static void transdd(int i, int j, int k, int dir, fab_t* qm, fab_t* qp, const fab_t* qnormm,
                    const fab_t* qnormp, const fab_t* flxx, const fab_t* flxy, const fab_t* qx,
                    const fab_t* qy, const fab_t* qa, const fab_t* srcq, double hdt, double cdtdx0,
                    double cdtdx1) {
  const int qvidx0 = (dir == 0) ? GDV : GDU;
  const int qvidx1 = (dir == 2) ? GDV : GDW;
  const int l1 = (dir == 0) ? 1 : 0;
  const int l2 = (dir == 2) ? 1 : 2;
  const int a1 = i + (l1 == 0), a2 = j + (l1 == 1), a3 = k + (l1 == 2); /* ivpt0 */
  const int b1 = i + (l2 == 0), b2 = j + (l2 == 1), b3 = k + (l2 == 2); /* ivpt1 */
  const int n1 = i + (dir == 0), n2 = j + (dir == 1), n3 = k + (dir == 2);
#define FD(c) (cdtdx0 * (F(*flxx, a1, a2, a3, c) - F(*flxx, i, j, k, c)) + \
               cdtdx1 * (F(*flxy, b1, b2, b3, c) - F(*flxy, i, j, k, c)))
  const double flxrho = FD(URHO);
  const double flxu = FD(UMX);
  const double flxv = FD(UMY);
  const double flxw = FD(UMZ);
  const double flxe = FD(UEDEN);
  const double c = F(*qa, i, j, k, QGAMC);
  const double srcrho = srcq ? F(*srcq, i, j, k, QRHO) : 0.0;
  const double srcu = srcq ? F(*srcq, i, j, k, QU) : 0.0;
  const double srcv = srcq ? F(*srcq, i, j, k, QV) : 0.0;
  const double srcw = srcq ? F(*srcq, i, j, k, QW) : 0.0;
  const double srce = srcq ? F(*srcq, i, j, k, QREINT) : 0.0;
  const double srcp = srcq ? F(*srcq, i, j, k, QPRES) : 0.0;
  const double rrr = F(*qnormp, i, j, k, QRHO);
  const double rrl = F(*qnormm, n1, n2, n3, QRHO);
  const double rrnewl = rrl - flxrho;
  const double rrnewr = rrr - flxrho;
  for (int n = 0; n < g_ns; n++) {
    const int uc = UFS + n, qc = QFS + n;
    const double srcpass = srcq ? F(*srcq, i, j, k, qc) : 0.0;
    const double compn = FD(uc);
    double compo = rrr * F(*qnormp, i, j, k, qc) - compn;
    F(*qp, i, j, k, qc) = compo / rrnewr + hdt * srcpass;
    compo = rrl * F(*qnormm, n1, n2, n3, qc) - compn;
    F(*qm, n1, n2, n3, qc) = compo / rrnewl + hdt * srcpass;
  }
#undef FD
  const double pggpx = F(*qx, a1, a2, a3, GDPRES);
  const double pggmx = F(*qx, i, j, k, GDPRES);
  const double ugpx = F(*qx, a1, a2, a3, qvidx0);
  const double ugmx = F(*qx, i, j, k, qvidx0);
  const double dAupx = pggpx * ugpx - pggmx * ugmx;
  const double pavx = 0.5 * (pggpx + pggmx);
  const double dAux = ugpx - ugmx;
  const double pggpy = F(*qy, b1, b2, b3, GDPRES);
  const double pggmy = F(*qy, i, j, k, GDPRES);
  const double ugpy = F(*qy, b1, b2, b3, qvidx1);
  const double ugmy = F(*qy, i, j, k, qvidx1);
  const double dAupy = pggpy * ugpy - pggmy * ugmy;
  const double pavy = 0.5 * (pggpy + pggmy);
  const double dAuy = ugpy - ugmy;
  const double pxnew = cdtdx0 * (dAupx + pavx * dAux * (c - 1.0));
  const double pynew = cdtdx1 * (dAupy + pavy * dAuy * (c - 1.0));
  {
    const double rur = rrr * F(*qnormp, i, j, k, QU);
    const double rvr = rrr * F(*qnormp, i, j, k, QV);
    const double rwr = rrr * F(*qnormp, i, j, k, QW);
    const double ekinr = 0.5 * (rur * rur + rvr * rvr + rwr * rwr) / rrr;
    const double rer = F(*qnormp, i, j, k, QREINT) + ekinr;
    const double runewr = rur - flxu;
    const double rvnewr = rvr - flxv;
    const double rwnewr = rwr - flxw;
    const double renewr = rer - flxe;
    F(*qp, i, j, k, QRHO) = rrnewr + hdt * srcrho;
    F(*qp, i, j, k, QU) = runewr / rrnewr + hdt * srcu;
    F(*qp, i, j, k, QV) = rvnewr / rrnewr + hdt * srcv;
    F(*qp, i, j, k, QW) = rwnewr / rrnewr + hdt * srcw;
    const double rhoekinr = 0.5 * (runewr * runewr + rvnewr * rvnewr + rwnewr * rwnewr) / rrnewr;
    F(*qp, i, j, k, QREINT) = renewr - rhoekinr + hdt * srce;
    F(*qp, i, j, k, QPRES) = F(*qnormp, i, j, k, QPRES) - pxnew - pynew + hdt * srcp;
    F(*qp, i, j, k, QPRES) = dmax(F(*qp, i, j, k, QPRES), DBL_MIN);
  }
  {
    const double rul = rrl * F(*qnormm, n1, n2, n3, QU);
    const double rvl = rrl * F(*qnormm, n1, n2, n3, QV);
    const double rwl = rrl * F(*qnormm, n1, n2, n3, QW);
    const double ekinl = 0.5 * (rul * rul + rvl * rvl + rwl * rwl) / rrl;
    const double rel = F(*qnormm, n1, n2, n3, QREINT) + ekinl;
    const double runewl = rul - flxu;
    const double rvnewl = rvl - flxv;
    const double rwnewl = rwl - flxw;
    const double renewl = rel - flxe;
    F(*qm, n1, n2, n3, QRHO) = rrnewl + hdt * srcrho;
    F(*qm, n1, n2, n3, QU) = runewl / rrnewl + hdt * srcu;
    F(*qm, n1, n2, n3, QV) = rvnewl / rrnewl + hdt * srcv;
    F(*qm, n1, n2, n3, QW) = rwnewl / rrnewl + hdt * srcw;
    const double rhoekinl = 0.5 * (runewl * runewl + rvnewl * rvnewl + rwnewl * rwnewl) / rrnewl;
    F(*qm, n1, n2, n3, QREINT) = renewl - rhoekinl + hdt * srce;
    F(*qm, n1, n2, n3, QPRES) = F(*qnormm, n1, n2, n3, QPRES) - pxnew - pynew + hdt * srcp;
    F(*qm, n1, n2, n3, QPRES) = dmax(F(*qm, n1, n2, n3, QPRES), DBL_MIN);
  }
}

/* ---------------------------------------------------------------- umeth */
/* Source/Godunov.cpp:6-55 (pc_low_order_boundary): the idir-fluxes on the face box bfbx
 * (one plane at a domain boundary) recomputed from PLM states of the two adjacent cells,
 * without transverse terms (the boundary state is given at time n). */
static void low_order_boundary(box_t bfbx, int bclo, int bchi, int domlo, int domhi, int plm_iorder,
                               int use_flattening, int idir, double dx, double dt, const fab_t* q,
                               const fab_t* qa, fab_t* flx, fab_t* qdir) {
  box_t bdbx = bfbx;
  bdbx.hi[idir] -= 1; /* enclosedCells */
  bdbx = bgrow_dir(bdbx, idir, 1);
  const box_t bdbx2 = bgrow_hi(bdbx, idir, 1);
  fab_t qbm = fab_new(bdbx2, QVAR), qbp = fab_new(bdbx, QVAR);
  double slope[MAXQ];
  FOR_BOX(bdbx, i, j, k) {
    double flat = 1.0;
    if (use_flattening)
      for (int df = 0; df < 3; df++) flat = dmin(flat, flatten(i, j, k, df, q));
    for (int n = 0; n < QVAR; ++n) slope[n] = plm_slope(i, j, k, n, idir, q, flat, plm_iorder);
    pc_plm_d(i, j, k, idir, &qbm, &qbp, slope, q, F(*qa, i, j, k, QC), dx, dt);
  }
  FOR_BOX(bfbx, i, j, k) cmpflx(i, j, k, bclo, bchi, domlo, domhi, &qbm, &qbp, flx, qdir, qa, idir);
  fab_free(&qbm);
  fab_free(&qbp);
}

/* Source/Godunov.cpp:59-476 (pc_umeth_3D), regular geometry. */
static int umeth_3d(box_t bx, const int* bclo, const int* bchi, const int* domlo, const int* domhi,
                    const fab_t* q, const fab_t* qaux, const fab_t* srcQ, fab_t* flx, fab_t* qec,
                    const fab_t* a, fab_t* pdivu, const fab_t* vol, const double* del, double dt,
                    int ppm_type, int plm_iorder, int use_flattening, int use_hybrid_weno, int weno_scheme) {
  const double dx = del[0], dy = del[1], dz = del[2];
  const double hdtdx = 0.5 * dt / dx, hdtdy = 0.5 * dt / dy, hdtdz = 0.5 * dt / dz;
  const double cdtdx = 1.0 / 3.0 * dt / dx, cdtdy = 1.0 / 3.0 * dt / dy, cdtdz = 1.0 / 3.0 * dt / dz;
  const double hdt = 0.5 * dt;
  const box_t bxg1 = bgrow(bx, 1), bxg2 = bgrow(bx, 2);
  fab_t qdm[3], qdp[3];
  box_t flxbx[3];
  for (int d = 0; d < 3; ++d) {
    qdm[d] = fab_new(bgrow_hi(bxg2, d, 1), QVAR);
    qdp[d] = fab_new(bxg2, QVAR);
    flxbx[d] = bnodes(bgrow_dir(bxg2, d, -1), d);
  }
  if (ppm_type == 0) {
    double slope[MAXQ];
    FOR_BOX(bxg2, i, j, k) {
      double flat = 1.0;
      if (use_flattening)
        for (int df = 0; df < 3; df++) flat = dmin(flat, flatten(i, j, k, df, q));
      for (int d = 0; d < 3; ++d) {
        for (int n = 0; n < QVAR; ++n) slope[n] = plm_slope(i, j, k, n, d, q, flat, plm_iorder);
        pc_plm_d(i, j, k, d, &qdm[d], &qdp[d], slope, q, F(*qaux, i, j, k, QC), del[d], dt);
      }
    }
  } else if (ppm_type == 1) {
    for (int d = 0; d < 3; ++d)
      trace_ppm(bxg2, d, q, &qdm[d], &qdp[d], dt, del, use_flattening, use_hybrid_weno, weno_scheme);
  } else {
    for (int d = 0; d < 3; ++d) { fab_free(&qdm[d]); fab_free(&qdp[d]); }
    return -2;
  }
  /* initial fluxes */
  fab_t f[3], gd[3];
  for (int d = 0; d < 3; ++d) {
    f[d] = fab_new(flxbx[d], NVAR);
    gd[d] = fab_new(flxbx[d], NGDNV);
    FOR_BOX(flxbx[d], i, j, k)
      cmpflx(i, j, k, bclo[d], bchi[d], domlo[d], domhi[d], &qdm[d], &qdp[d], &f[d], &gd[d], qaux, d);
  }
  const double cdt[3] = {cdtdx, cdtdy, cdtdz};
  /* transverse corrections and paired Riemann solves: flux fDO[d][o] is the d-flux
   * computed from d-states corrected by the o-flux. */
  fab_t fDO[3][3], gDO[3][3];
  for (int d = 0; d < 3; ++d) {
    const box_t tbx = bgrow_dir(bxg1, d, 1);
    const box_t tbxm = bgrow_hi(tbx, d, 1);
    const box_t tfbx = bnodes(bxg1, d);
    for (int o = 0; o < 3; ++o) {
      if (o == d) continue;
      fab_t tqm = fab_new(tbxm, QVAR), tqp = fab_new(tbx, QVAR);
      FOR_BOX(tbx, i, j, k)
        transdo(i, j, k, d, o, &tqm, &tqp, &qdm[d], &qdp[d], &f[o], qaux, &gd[o], cdt[o]);
      fDO[d][o] = fab_new(tfbx, NVAR);
      gDO[d][o] = fab_new(tfbx, NGDNV);
      FOR_BOX(tfbx, i, j, k)
        cmpflx(i, j, k, bclo[d], bchi[d], domlo[d], domhi[d], &tqm, &tqp, &fDO[d][o], &gDO[d][o], qaux, d);
      fab_free(&tqm);
      fab_free(&tqp);
    }
  }
  /* final fluxes: d-states corrected by fluxes (o1|o2) and (o2|o1) */
  fab_t qmf = fab_new(bxg2, QVAR), qpf = fab_new(bxg1, QVAR);
  const double hdtd[3] = {hdtdx, hdtdy, hdtdz};
  for (int d = 0; d < 3; ++d) {
    const int o1 = (d == 0) ? 1 : 0;
    const int o2 = (d == 2) ? 1 : 2;
    const box_t tbx = bgrow_dir(bx, d, 1);
    FOR_BOX(tbx, i, j, k)
      transdd(i, j, k, d, &qmf, &qpf, &qdm[d], &qdp[d], &fDO[o1][o2], &fDO[o2][o1], &gDO[o1][o2],
              &gDO[o2][o1], qaux, srcQ, hdt, hdtd[o1], hdtd[o2]);
    const box_t fbx = bnodes(bx, d);
    FOR_BOX(fbx, i, j, k)
      cmpflx(i, j, k, bclo[d], bchi[d], domlo[d], domhi[d], &qmf, &qpf, &flx[d], &qec[d], qaux, d);
  }
  /* Source/Godunov.cpp:440-468: faces on inflow / user_bc domain boundaries */
  for (int d = 0; d < 3; ++d) {
    if (bclo[d] == BC_INFLOW || bclo[d] == BC_USER) {
      box_t bfbx = bnodes(bx, d);
      bfbx.hi[d] = domlo[d];
      if (bfbx.lo[d] <= bfbx.hi[d])
        low_order_boundary(bfbx, bclo[d], bchi[d], domlo[d], domhi[d], plm_iorder, use_flattening, d, del[d], dt, q,
                           qaux, &flx[d], &qec[d]);
    }
    if (bchi[d] == BC_INFLOW || bchi[d] == BC_USER) {
      box_t bfbx = bnodes(bx, d);
      bfbx.lo[d] = domhi[d] + 1;
      if (bfbx.lo[d] <= bfbx.hi[d])
        low_order_boundary(bfbx, bclo[d], bchi[d], domlo[d], domhi[d], plm_iorder, use_flattening, d, del[d], dt, q,
                           qaux, &flx[d], &qec[d]);
    }
  }
  /* p div(u), Source/Godunov.H:1033-1060 */
  FOR_BOX(bx, i, j, k) {
    F(*pdivu, i, j, k, 0) =
      0.5 *
      ((F(qec[0], i + 1, j, k, GDPRES) + F(qec[0], i, j, k, GDPRES)) *
           (F(qec[0], i + 1, j, k, GDU) * F(a[0], i + 1, j, k, 0) - F(qec[0], i, j, k, GDU) * F(a[0], i, j, k, 0)) +
       (F(qec[1], i, j + 1, k, GDPRES) + F(qec[1], i, j, k, GDPRES)) *
           (F(qec[1], i, j + 1, k, GDV) * F(a[1], i, j + 1, k, 0) - F(qec[1], i, j, k, GDV) * F(a[1], i, j, k, 0)) +
       (F(qec[2], i, j, k + 1, GDPRES) + F(qec[2], i, j, k, GDPRES)) *
           (F(qec[2], i, j, k + 1, GDW) * F(a[2], i, j, k + 1, 0) - F(qec[2], i, j, k, GDW) * F(a[2], i, j, k, 0))) /
      F(*vol, i, j, k, 0);
  }
  for (int d = 0; d < 3; ++d) {
    fab_free(&qdm[d]); fab_free(&qdp[d]); fab_free(&f[d]); fab_free(&gd[d]);
    for (int o = 0; o < 3; ++o)
      if (o != d) { fab_free(&fDO[d][o]); fab_free(&gDO[d][o]); }
  }
  fab_free(&qmf);
  fab_free(&qpf);
  return 0;
}

/* ---------------------------------------------------------------- umdrv */
/* Source/Hydro.cpp:304-377 (pc_umdrv), :380-413 (pc_adjust_fluxes), :545-557 (pc_consup);
 * pointwise parts Source/Hydro.H:476-517 (pc_divu), Godunov.H:1067-1138 (pc_artif_visc),
 * Hydro.H:835-865 (pc_norm_spec_flx, pc_ext_flx), Hydro.H:888-907 (pc_update). */
int orc_umdrv(const orc_params* prm, const int32_t lo[3], const int32_t hi[3], const orc_array4* uin,
              orc_array4* uout, const orc_array4* q, const orc_array4* qaux, const orc_array4* srcq,
              orc_array4* flx, const orc_array4* area, const orc_array4* vol) {
  if (prm->nspec != g_ns) return -3;
  const box_t bx = mkbox(lo, hi);
  const box_t bxg2 = bgrow(bx, 2);
  fab_t uf = fab_view(uin), of = fab_view(uout), qf = fab_view(q), af = fab_view(qaux);
  fab_t sf, *sfp = NULL;
  if (srcq) { sf = fab_view(srcq); sfp = &sf; }
  fab_t ff[3], aa[3], qec[3];
  for (int d = 0; d < 3; ++d) {
    ff[d] = fab_view(&flx[d]);
    aa[d] = fab_view(&area[d]);
    qec[d] = fab_new(bnodes(bxg2, d), NGDNV);
  }
  fab_t vf = fab_view(vol);
  fab_t divu = fab_new(bxg2, 1), pdivu = fab_new(bx, 1);
  int rc = umeth_3d(bx, prm->bclo, prm->bchi, prm->domlo, prm->domhi, &qf, &af, sfp, ff, qec, aa, &pdivu,
                    &vf, prm->dx, prm->dt, prm->ppm_type, prm->plm_iorder, prm->use_flattening,
                    prm->use_hybrid_weno, prm->weno_scheme);
  if (rc == 0) {
    const double dx = prm->dx[0], dy = prm->dx[1], dz = prm->dx[2];
    FOR_BOX(bxg2, i, j, k) {
#define QQ(a, b, c, n) F(qf, a, b, c, n)
      double ux = 0.25 *
                  (QQ(i, j, k, QU) - QQ(i - 1, j, k, QU) + QQ(i, j, k - 1, QU) - QQ(i - 1, j, k - 1, QU) +
                   QQ(i, j - 1, k, QU) - QQ(i - 1, j - 1, k, QU) + QQ(i, j - 1, k - 1, QU) -
                   QQ(i - 1, j - 1, k - 1, QU)) /
                  dx;
      double vy = 0.25 *
                  (QQ(i, j, k, QV) - QQ(i, j - 1, k, QV) + QQ(i, j, k - 1, QV) - QQ(i, j - 1, k - 1, QV) +
                   QQ(i - 1, j, k, QV) - QQ(i - 1, j - 1, k, QV) + QQ(i - 1, j, k - 1, QV) -
                   QQ(i - 1, j - 1, k - 1, QV)) /
                  dy;
      double wz = 0.25 *
                  (QQ(i, j, k, QW) - QQ(i, j, k - 1, QW) + QQ(i - 1, j, k, QW) - QQ(i - 1, j, k - 1, QW) +
                   QQ(i, j - 1, k, QW) - QQ(i, j - 1, k - 1, QW) + QQ(i - 1, j - 1, k, QW) -
                   QQ(i - 1, j - 1, k - 1, QW)) /
                  dz;
#undef QQ
      F(divu, i, j, k, 0) = ux + vy + wz;
    }
    for (int d = 0; d < 3; ++d) {
      const box_t fbx = bnodes(bx, d);
      const double dxd = prm->dx[d];
      const int l1 = (d == 0) ? 1 : 0, l2 = (d == 2) ? 1 : 2;
      FOR_BOX(fbx, i, j, k) {
        /* pc_artif_visc */
        const int j1 = i + (l1 == 0), j2 = j + (l1 == 1), j3 = k + (l1 == 2);
        const int k1 = i + (l2 == 0), k2 = j + (l2 == 1), k3 = k + (l2 == 2);
        const int p1 = j1 + (l2 == 0), p2 = j2 + (l2 == 1), p3 = j3 + (l2 == 2);
        const double div = prm->difmag * dmin(0.0, 0.25 * (F(divu, i, j, k, 0) + F(divu, j1, j2, j3, 0) +
                                                           F(divu, k1, k2, k3, 0) + F(divu, p1, p2, p3, 0)));
        const int idx = (d == 0) ? i : (d == 1) ? j : k;
        const int at_bndry = (idx == prm->domlo[d] && prm->bclo[d] == BC_NO_SLIP_WALL) ||
                             (idx == prm->domhi[d] + 1 && prm->bchi[d] == BC_NO_SLIP_WALL);
        const int m1 = i - (d == 0), m2 = j - (d == 1), m3 = k - (d == 2);
        for (int n = 0; n < NVAR; n++) {
          if (n == UTEMP) continue;
          const int is_tang = (d == 0 && (n == UMY || n == UMZ)) || (d == 1 && (n == UMX || n == UMZ)) ||
                              (d == 2 && (n == UMX || n == UMY));
          if (!(at_bndry && is_tang))
            F(ff[d], i, j, k, n) += dxd * div * (F(uf, i, j, k, n) - F(uf, m1, m2, m3, n));
        }
        F(ff[d], i, j, k, UTEMP) = 0.0;
        /* pc_norm_spec_flx */
        double summ = 0.0;
        for (int n = UFS; n < UFS + g_ns; ++n) summ += F(ff[d], i, j, k, n);
        const double fac = (summ != 0.0) ? F(ff[d], i, j, k, URHO) / summ : 1.0;
        for (int n = UFS; n < UFS + g_ns; ++n) F(ff[d], i, j, k, n) *= fac;
        /* pc_ext_flx */
        const double ar = F(aa[d], i, j, k, 0);
        for (int n = 0; n < NVAR; ++n) F(ff[d], i, j, k, n) *= ar;
      }
    }
    FOR_BOX(bx, i, j, k) {
      const double v = F(vf, i, j, k, 0);
      for (int n = 0; n < NVAR; ++n) {
        F(of, i, j, k, n) += (F(ff[0], i, j, k, n) - F(ff[0], i + 1, j, k, n) + F(ff[1], i, j, k, n) -
                              F(ff[1], i, j + 1, k, n) + F(ff[2], i, j, k, n) - F(ff[2], i, j, k + 1, n)) /
                             v;
      }
      F(of, i, j, k, UEINT) -= F(pdivu, i, j, k, 0);
    }
  }
  for (int d = 0; d < 3; ++d) fab_free(&qec[d]);
  fab_free(&divu);
  fab_free(&pdivu);
  return rc;
}

/* Source/Hydro.cpp:70-249 for one regular box, no sources (sources_for_hydro == 0). */
int orc_hydro_box(const orc_params* prm, const int32_t lo[3], const int32_t hi[3], const orc_array4* uin,
                  orc_array4* uout, orc_array4* flx, const orc_array4* area, const orc_array4* vol) {
  if (prm->nspec != g_ns) return -3;
  const box_t bx = mkbox(lo, hi);
  const box_t qbx = bgrow(bx, 4);
  fab_t q = fab_new(qbx, QVAR), qa = fab_new(qbx, NQAUX), sq = fab_new(qbx, QVAR);
  fab_t uf = fab_view(uin);
  FOR_BOX(qbx, i, j, k) ctoprim_cell(i, j, k, &uf, &q, &qa);
  fab_t zero_src = fab_new(qbx, NVAR);
  FOR_BOX(qbx, i, j, k) srctoprim_cell(i, j, k, &q, &qa, &zero_src, &sq);
  fab_free(&zero_src);
  /* hydro_source.setVal(0) (Hydro.cpp:47) and flux[dir].setVal(0) (:88) */
  fab_t of = fab_view(uout);
  FOR_BOX(bx, i, j, k) for (int n = 0; n < NVAR; ++n) F(of, i, j, k, n) = 0.0;
  for (int d = 0; d < 3; ++d) {
    fab_t ff = fab_view(&flx[d]);
    const box_t fbx = bnodes(bx, d);
    FOR_BOX(fbx, i, j, k) for (int n = 0; n < NVAR; ++n) F(ff, i, j, k, n) = 0.0;
  }
  orc_array4 qv = {q.p, q.js, q.ks, q.ns, {qbx.lo[0], qbx.lo[1], qbx.lo[2]},
                   {qbx.hi[0] + 1, qbx.hi[1] + 1, qbx.hi[2] + 1}, QVAR};
  orc_array4 av = {qa.p, qa.js, qa.ks, qa.ns, {qbx.lo[0], qbx.lo[1], qbx.lo[2]},
                   {qbx.hi[0] + 1, qbx.hi[1] + 1, qbx.hi[2] + 1}, NQAUX};
  orc_array4 sv = {sq.p, sq.js, sq.ks, sq.ns, {qbx.lo[0], qbx.lo[1], qbx.lo[2]},
                   {qbx.hi[0] + 1, qbx.hi[1] + 1, qbx.hi[2] + 1}, QVAR};
  int rc = orc_umdrv(prm, lo, hi, uin, uout, &qv, &av, &sv, flx, area, vol);
  fab_free(&q);
  fab_free(&qa);
  fab_free(&sq);
  return rc;
}

/* Source/Hydro.cpp:161-174: pc_srctoprim (Source/Hydro.H:14-68) over a box. */
int orc_srctoprim(const int32_t lo[3], const int32_t hi[3], const orc_array4* q, const orc_array4* qaux,
                  const orc_array4* src, orc_array4* srcq) {
  fab_t qf = fab_view(q), af = fab_view(qaux), sf = fab_view(src), of = fab_view(srcq);
  box_t b = mkbox(lo, hi);
  FOR_BOX(b, i, j, k) srctoprim_cell(i, j, k, &qf, &af, &sf, &of);
  return 0;
}

/* pc_umeth_3D (Source/Godunov.cpp:59-476, declared Source/Godunov.H:1142-1162) on its own:
 * flx[d] receives the final Godunov fluxes on the d-faces of the box (before the
 * artificial viscosity, species normalisation and area weighting of pc_adjust_fluxes),
 * qec[d] the face states GDU, GDV, GDW, GDPRES, GDGAME (GDRHO is not written, as in the
 * reference), pdivu the cell-centred p div u. srcq may be NULL (no sources). */
int orc_umeth(const orc_params* prm, const int32_t lo[3], const int32_t hi[3], const orc_array4* q,
              const orc_array4* qaux, const orc_array4* srcq, orc_array4* flx, orc_array4* qec,
              const orc_array4* area, orc_array4* pdivu, const orc_array4* vol) {
  if (prm->nspec != g_ns) return -3;
  const box_t bx = mkbox(lo, hi);
  fab_t qf = fab_view(q), af = fab_view(qaux), pf = fab_view(pdivu), vf = fab_view(vol);
  fab_t sf, *sfp = NULL;
  if (srcq) { sf = fab_view(srcq); sfp = &sf; }
  fab_t ff[3], gf[3], aa[3];
  for (int d = 0; d < 3; ++d) {
    ff[d] = fab_view(&flx[d]);
    gf[d] = fab_view(&qec[d]);
    aa[d] = fab_view(&area[d]);
  }
  return umeth_3d(bx, prm->bclo, prm->bchi, prm->domlo, prm->domhi, &qf, &af, sfp, ff, gf, aa, &pf, &vf, prm->dx,
                  prm->dt, prm->ppm_type, prm->plm_iorder, prm->use_flattening, prm->use_hybrid_weno,
                  prm->weno_scheme);
}

/* ---------------------------------------------------------------- timestep */
/* Source/Timestep.H:51-88 (pc_estdt_hydro), regular cells. */
double orc_estdt(const int32_t lo[3], const int32_t hi[3], const orc_array4* u, const double dx[3]) {
  fab_t uf = fab_view(u);
  box_t b = mkbox(lo, hi);
  double dt = DBL_MAX;
  FOR_BOX(b, i, j, k) {
    const double rho = F(uf, i, j, k, URHO);
    const double rhoInv = 1.0 / rho;
    double T = F(uf, i, j, k, UTEMP);
    double massfrac[ORC_MAXNS];
    double c;
    for (int n = 0; n < g_ns; ++n) massfrac[n] = F(uf, i, j, k, UFS + n) * rhoInv;
    orc_eos_rty2cs(rho, T, massfrac, &c);
    const double ux = F(uf, i, j, k, UMX) * rhoInv;
    const double dt1 = dx[0] / (c + fabs(ux));
    dt = dmin(dt, dt1);
    const double uy = F(uf, i, j, k, UMY) * rhoInv;
    const double dt2 = dx[1] / (c + fabs(uy));
    dt = dmin(dt, dt2);
    const double uz = F(uf, i, j, k, UMZ) * rhoInv;
    const double dt3 = dx[2] / (c + fabs(uz));
    dt = dmin(dt, dt3);
  }
  return dt;
}

/* Source/Advance.cpp:397-417 (construct_Snew, hydro only), then Source/PeleC.cpp:2289-2305
 * (computeTemp): pc_rst_int_e default branch (PeleCUtilities.H:227-235, allow_small_energy
 * and allow_negative_energy true) and pc_cmpTemp (PeleCUtilities.H:70-84). */
int orc_update_state(const int32_t lo[3], const int32_t hi[3], const orc_array4* s_old,
                     const orc_array4* hydro_source, double dt, orc_array4* s_new) {
  fab_t so = fab_view(s_old), hs = fab_view(hydro_source), sn = fab_view(s_new);
  box_t b = mkbox(lo, hi);
  FOR_BOX(b, i, j, k) {
    for (int n = 0; n < NVAR; ++n) {
      F(sn, i, j, k, n) = F(so, i, j, k, n);
      F(sn, i, j, k, n) += dt * F(hs, i, j, k, n);
    }
    const double rho = F(sn, i, j, k, URHO);
    const double rhoInv = 1.0 / rho;
    const double Up = F(sn, i, j, k, UMX) * rhoInv;
    const double Vp = F(sn, i, j, k, UMY) * rhoInv;
    const double Wp = F(sn, i, j, k, UMZ) * rhoInv;
    const double ke = 0.5 * (Up * Up + Vp * Vp + Wp * Wp) - 0.5 * 0.0 * 0.0 * 0.0 * 0.0;
    F(sn, i, j, k, UEINT) = F(sn, i, j, k, UEDEN) - rho * ke;
    const double rhoInv2 = 1.0 / F(sn, i, j, k, URHO);
    double T = F(sn, i, j, k, UTEMP);
    const double e = F(sn, i, j, k, UEINT) * rhoInv2;
    double massfrac[ORC_MAXNS];
    for (int n = 0; n < g_ns; ++n) massfrac[n] = F(sn, i, j, k, UFS + n) * rhoInv2;
    orc_eos_rey2t(F(sn, i, j, k, URHO), e, massfrac, &T);
    F(sn, i, j, k, UTEMP) = T;
  }
  return 0;
}
