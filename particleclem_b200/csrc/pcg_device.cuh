// pcg_device.cuh -- pointwise device code of the Godunov hydro advance.
//
// Every function restates the reference routine it names (paths relative to the
// reference project root) with the same operation order. The compute type R is
// double for the FP64 forms and float for the mixed form's trace / Riemann /
// transverse arithmetic. In the FP64 parity build (translation unit compiled with
// --fmad=false) the results are bit-identical to the CPU oracle.
#pragma once

#include <cfloat>
#include <cstdint>

#include "pcg_types.h"

namespace PCG_TU {

// ------------------------------------------------------------------ constants
template <class R> struct Lim;
template <> struct Lim<double> {
  static __device__ __forceinline__ double tiny() { return DBL_MIN; }
  static __device__ __forceinline__ double eps() { return DBL_EPSILON; }
  // constants::very_small_num() and flatten's small_pres (Source/Constants.H:28-31,
  // Source/Godunov.H:208); in FP32 they underflow, so the smallest normal is used.
  static __device__ __forceinline__ double very_small() { return pcg::VERY_SMALL_NUM; }
  static __device__ __forceinline__ double small_pres() { return 1.e-200; }
};
template <> struct Lim<float> {
  static __device__ __forceinline__ float tiny() { return FLT_MIN; }
  static __device__ __forceinline__ float eps() { return FLT_EPSILON; }
  static __device__ __forceinline__ float very_small() { return FLT_MIN; }
  static __device__ __forceinline__ float small_pres() { return FLT_MIN; }
};

// amrex::min / amrex::max are std::min / std::max
template <class R> __device__ __forceinline__ R dmin(R a, R b) { return (b < a) ? b : a; }
template <class R> __device__ __forceinline__ R dmax(R a, R b) { return (a < b) ? b : a; }

// The reference's clamps to [0, 1], nested std::min/std::max, including their results
// for NaN: max(0, min(1, NaN)) is 1 and min(1, max(0, NaN)) is 0. The NaN case is
// written out because the device compiler folds a nested min/max into a saturating
// clamp, which maps NaN to 0 in both orders.
template <class R> __device__ __forceinline__ R max0_min1(R x) { return (x != x) ? R(1) : dmax(R(0), dmin(R(1), x)); }
template <class R> __device__ __forceinline__ R min1_max0(R x) { return (x != x) ? R(0) : dmin(R(1), dmax(R(0), x)); }

// Pressure in the FP32 arithmetic is carried as the deviation p' = p - p0 from a
// constant p0 of the box (rho*R/W*T of its first cell): PPM/PLM reconstruction, the
// characteristic projection, the linearised star state and the flux differences are
// invariant under a constant pressure shift, so only the EOS calls (which take p0 + p')
// and the transverse pressure terms (which gain p0 * gamma_c * du) see p0. In FP64 the
// pressure is absolute (p0 = 0) and these helpers are the identity.
template <class R> struct PDev { static constexpr bool on = sizeof(R) == 4; };
template <class R> __device__ __forceinline__ R pabs(R pdev, R p0) {
  if constexpr (PDev<R>::on) return pdev + p0; else return pdev;
}
// floor of the deviation equivalent to the floor f of the absolute pressure
template <class R> __device__ __forceinline__ R pfloor(R f, R p0) {
  if constexpr (PDev<R>::on) return f - p0; else return f;
}

// ------------------------------------------------------------------ views
// Element offsets within one view are 32-bit: the host refuses arrays whose component
// extent (ncomp * nstride) or strides reach 2^31 elements (pcg::kMaxViewElems), so every
// address is one 32-bit index computation and one scaled add to the 64-bit base, instead
// of 64-bit multiply-adds per component (the flux stages' address arithmetic was about a
// third of their instructions with 64-bit offsets).
template <class T>
struct V4 {
  T* p;
  int js, ks, ns;
  int bx, by, bz;
  __device__ __forceinline__ T& operator()(int i, int j, int k, int n = 0) const {
    return p[(i - bx) + (j - by) * js + (k - bz) * ks + n * ns];
  }
};
template <class T>
__device__ __forceinline__ V4<T> v4(const pcg::View& w) {
  return V4<T>{reinterpret_cast<T*>(w.p), (int)w.js, (int)w.ks, (int)w.ns, w.b[0], w.b[1], w.b[2]};
}

// A view of a blocked workspace array (pcg::View::blocked, pcg::kCellBlock): cell(i, j, k)
// is the address of component 0 of the cell; component n is kCellBlock * n elements on.
template <class T>
struct B4 {
  T* p;
  int js, ks, bs;
  int bx, by, bz;
  __device__ __forceinline__ T* cell(int i, int j, int k) const {
    const int L = (i - bx) + (j - by) * js + (k - bz) * ks;
    return p + ((L >> 5) * bs + (L & (pcg::kCellBlock - 1)));
  }
  __device__ __forceinline__ T& operator()(int i, int j, int k, int n = 0) const {
    return cell(i, j, k)[n * pcg::kCellBlock];
  }
};
template <class T>
__device__ __forceinline__ B4<T> b4(const pcg::View& w) {
  return B4<T>{reinterpret_cast<T*>(w.p), (int)w.js, (int)w.ks, (int)w.ns, w.b[0], w.b[1], w.b[2]};
}

// ------------------------------------------------------------------ EOS
// PelePhysics' eos() restated (documented in the oracle): rmix = RU * sum Y_k / W_k;
// gamma law: cs = sqrt(gamma P / R), e = P / ((gamma-1) R); NASA-7 mixture:
// T = P / (R rmix), cv = sum Y_k cv_k(T), e = sum Y_k e_k(T), G = (cv + rmix) / cv.
// slot 0: gamma law (one species), slot 1: NASA-7 mixture
__constant__ pcg::EosConst c_eos[2];  // one bank per translation unit

template <class R> __device__ __forceinline__ R eos_ru();
template <> __device__ __forceinline__ double eos_ru<double>() { return pcg::RU; }
template <> __device__ __forceinline__ float eos_ru<float>() { return (float)pcg::RU; }

template <class R, bool MIX> struct EosC;
template <bool MIX> struct EosC<double, MIX> {
  static __device__ __forceinline__ const pcg::EosConst& e() { return c_eos[MIX ? 1 : 0]; }
  static __device__ __forceinline__ bool uniform_tmid() { return e().uniform_tmid != 0; }
  static __device__ __forceinline__ double cvr(int k, int r, int i) { return e().cvc[k][r][i]; }
  static __device__ __forceinline__ double ecr(int k, int r, int i) { return e().ec[k][r][i]; }
  static __device__ __forceinline__ double gamma() { return e().gamma; }
  static __device__ __forceinline__ double imw(int k) { return e().imw[k]; }
  static __device__ __forceinline__ double tmid(int k) { return e().tmid[k]; }
  static __device__ __forceinline__ const double* cv(int k, int r) { return e().cvc[k][r]; }
  static __device__ __forceinline__ const double* ec(int k, int r) { return e().ec[k][r]; }
};
template <bool MIX> struct EosC<float, MIX> {
  static __device__ __forceinline__ const pcg::EosConst& e() { return c_eos[MIX ? 1 : 0]; }
  static __device__ __forceinline__ bool uniform_tmid() { return e().uniform_tmid != 0; }
  static __device__ __forceinline__ float cvr(int k, int r, int i) { return e().cvcf[k][r][i]; }
  static __device__ __forceinline__ float ecr(int k, int r, int i) { return e().ecf[k][r][i]; }
  static __device__ __forceinline__ float gamma() { return e().gammaf; }
  static __device__ __forceinline__ float imw(int k) { return e().imwf[k]; }
  static __device__ __forceinline__ float tmid(int k) { return e().tmidf[k]; }
  static __device__ __forceinline__ const float* cv(int k, int r) { return e().cvcf[k][r]; }
  static __device__ __forceinline__ const float* ec(int k, int r) { return e().ecf[k][r]; }
};

// Species sums of the FP32 mixture EOS with Blackwell's packed FP32 arithmetic (FFMA2,
// two lanes per instruction): species 2m and 2m+1 share one instruction, their
// coefficients one aligned pair of the species-minor rows (EosConst::cvp/ecp/imwp).
// The even and odd species accumulate separately and meet at the end, so the order of
// the additions differs from the scalar sums (well inside the mixed form's tolerance).
__device__ __forceinline__ float2 cpair(const float* row, int k) { return *reinterpret_cast<const float2*>(row + k); }
// sum_k y_k * P_k(t), P_k the degree NC-1 polynomial with coefficients rows[i][k]
template <int NS, int NC>
__device__ __forceinline__ float poly_sum_f2(float t, const float* y, const float (*rows)[pcg::MAXNS]) {
  const float2 t2 = make_float2(t, t);
  float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int m = 0; m < NS / 2; ++m) {
    float2 c = cpair(rows[NC - 1], 2 * m);
#pragma unroll
    for (int i = NC - 2; i >= 0; --i) c = __ffma2_rn(t2, c, cpair(rows[i], 2 * m));
    acc = __ffma2_rn(make_float2(y[2 * m], y[2 * m + 1]), c, acc);
  }
  float s = acc.x + acc.y;
  if constexpr (NS % 2) {
    float c = rows[NC - 1][NS - 1];
#pragma unroll
    for (int i = NC - 2; i >= 0; --i) c = fmaf(t, c, rows[i][NS - 1]);
    s = fmaf(y[NS - 1], c, s);
  }
  return s;
}
// sum_k y_k * w[k]
template <int NS>
__device__ __forceinline__ float wsum_f2(const float* y, const float* w) {
  float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int m = 0; m < NS / 2; ++m) acc = __ffma2_rn(make_float2(y[2 * m], y[2 * m + 1]), cpair(w, 2 * m), acc);
  float s = acc.x + acc.y;
  if constexpr (NS % 2) s = fmaf(y[NS - 1], w[NS - 1], s);
  return s;
}

// Species loops of the FP32 form in packed pairs: a[n] = ca * x[n] + cb * y[n] for
// n < N (two species per FFMA2/FMUL2), returning the sum of the a[n].
template <int N>
__device__ __forceinline__ float blend2_sum(float ca, const float* x, float cb, const float* y, float* a) {
  const float2 ca2 = make_float2(ca, ca), cb2 = make_float2(cb, cb);
  float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int m = 0; m < N / 2; ++m) {
    const float2 v = __ffma2_rn(ca2, make_float2(x[2 * m], x[2 * m + 1]),
                                __fmul2_rn(cb2, make_float2(y[2 * m], y[2 * m + 1])));
    a[2 * m] = v.x;
    a[2 * m + 1] = v.y;
    acc = __fadd2_rn(acc, v);
  }
  float s = acc.x + acc.y;
  if constexpr (N % 2) {
    a[N - 1] = fmaf(ca, x[N - 1], cb * y[N - 1]);
    s += a[N - 1];
  }
  return s;
}
// a[n] = (r * q[n] - c[n]) * inv for n < N, in packed pairs
template <int N>
__device__ __forceinline__ void scale_sub2(float r, const float* q, const float* c, float inv, float* a) {
  const float2 r2 = make_float2(r, r), i2 = make_float2(inv, inv);
#pragma unroll
  for (int m = 0; m < N / 2; ++m) {
    const float2 v = __ffma2_rn(r2, make_float2(q[2 * m], q[2 * m + 1]), make_float2(-c[2 * m], -c[2 * m + 1]));
    const float2 w = __fmul2_rn(v, i2);
    a[2 * m] = w.x;
    a[2 * m + 1] = w.y;
  }
  if constexpr (N % 2) a[N - 1] = fmaf(r, q[N - 1], -c[N - 1]) * inv;
}

template <int NS, bool MIX, class R>
struct Eos {
  using C = EosC<R, MIX>;
  static __device__ __forceinline__ R rmix(const R* y) {
    if constexpr (sizeof(R) == 4 && NS > 1) return eos_ru<R>() * wsum_f2<NS>(y, C::e().imwp);
    R s = R(0);
#pragma unroll
    for (int k = 0; k < NS; ++k) s = s + y[k] * C::imw(k);
    return eos_ru<R>() * s;
  }
  // Species polynomials; both temperature ranges are loaded (warp-uniform constant
  // addresses) and the range is selected per thread.
  static __device__ __forceinline__ R cv_k(int k, R t) {
    const R* a = C::cv(k, 0);
    const R* b = C::cv(k, 1);
    const bool lo = t < C::tmid(k);
    const R c0 = lo ? a[0] : b[0], c1 = lo ? a[1] : b[1], c2 = lo ? a[2] : b[2], c3 = lo ? a[3] : b[3],
            c4 = lo ? a[4] : b[4];
    return c0 + t * (c1 + t * (c2 + t * (c3 + t * c4)));
  }
  static __device__ __forceinline__ R e_k(int k, R t) {
    const R* a = C::ec(k, 0);
    const R* b = C::ec(k, 1);
    const bool lo = t < C::tmid(k);
    const R c0 = lo ? a[0] : b[0], c1 = lo ? a[1] : b[1], c2 = lo ? a[2] : b[2], c3 = lo ? a[3] : b[3],
            c4 = lo ? a[4] : b[4], c5 = lo ? a[5] : b[5];
    return c0 + t * (c1 + t * (c2 + t * (c3 + t * (c4 + t * c5))));
  }
  // With one range switch temperature for all species the range is chosen once per
  // call and every coefficient is a compile-time constant-bank operand (no indexed
  // constant loads); the arithmetic is identical to the per-species selection.
  template <int RG>
  static __device__ __forceinline__ R cv_sum(R t, const R* y) {
    if constexpr (sizeof(R) == 4 && NS > 1) return poly_sum_f2<NS, 5>(t, y, C::e().cvp[RG]);
    R cv = R(0);
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const R cvk = C::cvr(k, RG, 0) + t * (C::cvr(k, RG, 1) + t * (C::cvr(k, RG, 2) + t * (C::cvr(k, RG, 3) + t * C::cvr(k, RG, 4))));
      cv = cv + y[k] * cvk;
    }
    return cv;
  }
  template <int RG>
  static __device__ __forceinline__ R e_sum(R t, const R* y) {
    if constexpr (sizeof(R) == 4 && NS > 1) return poly_sum_f2<NS, 6>(t, y, C::e().ecp[RG]);
    R e = R(0);
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const R ek = C::ecr(k, RG, 0) + t * (C::ecr(k, RG, 1) + t * (C::ecr(k, RG, 2) + t * (C::ecr(k, RG, 3) + t * (C::ecr(k, RG, 4) + t * C::ecr(k, RG, 5)))));
      e = e + y[k] * ek;
    }
    return e;
  }
  static __device__ __forceinline__ R cv_of(R t, const R* y) {
    if (C::uniform_tmid()) return (t < C::tmid(0)) ? cv_sum<0>(t, y) : cv_sum<1>(t, y);
    R cv = R(0);
#pragma unroll
    for (int k = 0; k < NS; ++k) cv = cv + y[k] * cv_k(k, t);
    return cv;
  }
  static __device__ __forceinline__ R e_of(R t, const R* y) {
    if (C::uniform_tmid()) return (t < C::tmid(0)) ? e_sum<0>(t, y) : e_sum<1>(t, y);
    R e = R(0);
#pragma unroll
    for (int k = 0; k < NS; ++k) e = e + y[k] * e_k(k, t);
    return e;
  }
  // RPY2Cs
  static __device__ __forceinline__ R rpy2cs(R r, R p, const R* y) {
    if (!MIX) return sqrt(C::gamma() * p / r);
    const R rm = rmix(y);
    const R t = p / (r * rm);
    const R cv = cv_of(t, y);
    const R g = (cv + rm) / cv;
    return sqrt(g * p / r);
  }
  // RYP2E
  static __device__ __forceinline__ R ryp2e(R r, const R* y, R p) {
    if (!MIX) return p / ((C::gamma() - R(1)) * r);
    const R rm = rmix(y);
    const R t = p / (r * rm);
    return e_of(t, y);
  }
  // REY2T (Newton from the stored temperature for the mixture)
  static __device__ __forceinline__ R rey2t(R e, const R* y, R tguess) {
    const R rm = rmix(y);
    if (!MIX) return e * (C::gamma() - R(1)) / rm;
    R tt = tguess;
    if (!(tt > R(0))) tt = R(1000);
    for (int it = 0; it < pcg::NEWTON_MAXIT; ++it) {
      const R ek = e_of(tt, y);
      const R cvk = cv_of(tt, y);
      const R dt = (e - ek) / cvk;
      tt = tt + dt;
      if (tt < R(pcg::NEWTON_TMIN)) tt = R(pcg::NEWTON_TMIN);
      if (fabs(dt) <= R(pcg::NEWTON_RTOL) * tt) break;
    }
    return tt;
  }
  static __device__ __forceinline__ R rty2p(R r, R t, const R* y) { return r * rmix(y) * t; }
  static __device__ __forceinline__ R rty2cs(R r, R t, const R* y) {
    const R rm = rmix(y);
    const R p = r * rm * t;
    if (!MIX) return sqrt(C::gamma() * p / r);
    const R cv = cv_of(t, y);
    const R g = (cv + rm) / cv;
    return sqrt(g * p / r);
  }
  static __device__ __forceinline__ R rty2g(R t, const R* y) {
    if (!MIX) return C::gamma();
    const R cv = cv_of(t, y);
    return (cv + rmix(y)) / cv;
  }
  static __device__ __forceinline__ void rty2dpde_dpdre(R r, R t, const R* y, R& dpde, R& dpdr_e) {
    const R rm = rmix(y);
    if (!MIX) {
      dpde = (C::gamma() - R(1)) * r;
    } else {
      dpde = r * rm / cv_of(t, y);
    }
    dpdr_e = rm * t;
  }
  // RTY2P, RTY2Cs, RTY2G and RTY2dpde_dpdre of one state, sharing rmix and cv: each
  // value is formed by exactly the operations of the separate calls.
  static __device__ __forceinline__ void rty2all(R r, R t, const R* y, R& p, R& cs, R& g, R& dpde, R& dpdr_e) {
    const R rm = rmix(y);
    p = r * rm * t;
    if (!MIX) {
      g = C::gamma();
      cs = sqrt(C::gamma() * p / r);
      dpde = (C::gamma() - R(1)) * r;
    } else {
      const R cv = cv_of(t, y);
      g = (cv + rm) / cv;
      cs = sqrt(g * p / r);
      dpde = r * rm / cv;
    }
    dpdr_e = rm * t;
  }
  static __device__ __forceinline__ R y2wbar(const R* y) {
    R s = R(0);
#pragma unroll
    for (int k = 0; k < NS; ++k) s = s + y[k] * C::imw(k);
    return R(1) / s;
  }
};

// ------------------------------------------------------------------ reduced EOS algebra
// The FMA and mixed forms evaluate the same EOS with fewer divisions, using that the
// restated EOS is linear in the mass fractions: for partial densities w_k (sum rho),
//   rmix = RU * sum(w_k / W_k) / rho,   T(rho, p) = p / (RU * sum(w_k / W_k)),
//   rho * cv = sum(w_k cv_k(T)),        rho * e = sum(w_k e_k(T)),
//   c^2 = (1 + RU * sum(w_k / W_k) / sum(w_k cv_k(T))) * p / rho.
// Results differ from the reference expressions only by rounding.
template <class R> __device__ __forceinline__ R rdiv(R a, R b) { return a / b; }
template <> __device__ __forceinline__ float rdiv<float>(float a, float b) { return __fdividef(a, b); }
template <class R> __device__ __forceinline__ R rrcp(R a) { return R(1) / a; }
template <> __device__ __forceinline__ float rrcp<float>(float a) { return __fdividef(1.0f, a); }

template <int NS, bool MIX, class R>
struct EosR {
  using E = Eos<NS, MIX, R>;
  using C = EosC<R, MIX>;
  static __device__ __forceinline__ R sum_imw(const R* w) {
    if constexpr (sizeof(R) == 4 && NS > 1) return wsum_f2<NS>(w, C::e().imwp);
    R s = R(0);
#pragma unroll
    for (int k = 0; k < NS; ++k) s = s + w[k] * C::imw(k);
    return s;
  }
  // sound speed from density r, pressure p and mass fractions y (RPY2Cs)
  static __device__ __forceinline__ R cs_y(R r, R p, const R* y) {
    if (!MIX) return sqrt(rdiv(C::gamma() * p, r));
    const R rus = eos_ru<R>() * sum_imw(y);
    const R t = rdiv(p, rus * r);
    return sqrt(rdiv((R(1) + rdiv(rus, E::cv_of(t, y))) * p, r));
  }
  // sound speed from pressure p and partial densities w (sum r)
  static __device__ __forceinline__ R cs_w(R r, R p, const R* w) {
    if (!MIX) return sqrt(rdiv(C::gamma() * p, r));
    const R rus = eos_ru<R>() * sum_imw(w);
    const R t = rdiv(p, rus);
    return sqrt(rdiv((R(1) + rdiv(rus, E::cv_of(t, w))) * p, r));
  }
  // rho * e from density r, pressure p and mass fractions y (r * RYP2E)
  static __device__ __forceinline__ R rhoe_y(R r, R p, const R* y) {
    if (!MIX) return p * rrcp(C::gamma() - R(1));
    const R t = rdiv(p, eos_ru<R>() * sum_imw(y) * r);
    return r * E::e_of(t, y);
  }
  // rho * e from pressure p and partial densities w
  static __device__ __forceinline__ R rhoe_w(R p, const R* w) {
    if (!MIX) return p * rrcp(C::gamma() - R(1));
    const R t = rdiv(p, eos_ru<R>() * sum_imw(w));
    return E::e_of(t, w);
  }
};

// ------------------------------------------------------------------ hybrid WENO
// Source/WENO.H: edge values of the centre cell of a stencil (sm on its low face, sp on
// its high face) replacing the PPM parabola when use_hybrid_weno is set
// (Source/PPM.cpp:120-172): WENO-JS5 (Jiang & Shu 1996), WENO-Z5 (Borges et al. 2008),
// WENO-Z7 (Balsara & Shu 2000 stencils, Z weights), WENO-Z3. Each expression keeps the
// reference's operation order (pow(x, 2) is x * x), so the FP64 form is bit-identical.
namespace weno {
template <class R> __device__ __forceinline__ R sq(R x) { return x * x; }
template <class R> __device__ __forceinline__ R eps() { return R(1e-6); }

template <class R>
__device__ __forceinline__ void w_weights(R* b, int n, R tau, bool z) {
#pragma unroll
  for (int m = 0; m < 4; ++m)
    if (m < n)
      b[m] = z ? R(1) + (tau / (eps<R>() + b[m])) * (tau / (eps<R>() + b[m]))
               : R(1) / ((eps<R>() + b[m]) * (eps<R>() + b[m]));
}
template <class R>
__device__ __forceinline__ R w5_blend(const R* b, const R* v) {
  const R a2 = b[2], a1 = R(6) * b[1], a0 = R(3) * b[0];
  const R ai = R(1) / (a2 + a1 + a0);
  return R(1.0 / 6.0) * ai * (a2 * v[2] + a1 * v[1] + a0 * v[0]);
}
template <class R>
__device__ __forceinline__ void weno5(const R* s, bool z, R& sm, R& sp) {
  const R k13 = R(13.0 / 12.0);
  R b[3], v[3];
  b[2] = k13 * sq(s[0] - R(2) * s[1] + s[2]) + R(0.25) * sq(s[0] - R(4) * s[1] + R(3) * s[2]);
  b[1] = k13 * sq(s[1] - R(2) * s[2] + s[3]) + R(0.25) * (s[1] - s[3]) * (s[1] - s[3]);
  b[0] = k13 * sq(s[2] - R(2) * s[3] + s[4]) + R(0.25) * sq(R(3) * s[2] - R(4) * s[3] + s[4]);
  w_weights(b, 3, fabs(b[2] - b[0]), z);
  v[2] = R(2) * s[0] - R(7) * s[1] + R(11) * s[2];
  v[1] = -s[1] + R(5) * s[2] + R(2) * s[3];
  v[0] = R(2) * s[2] + R(5) * s[3] - s[4];
  sp = w5_blend(b, v);
  b[2] = k13 * sq(s[4] - R(2) * s[3] + s[2]) + R(0.25) * sq(s[4] - R(4) * s[3] + R(3) * s[2]);
  b[1] = k13 * sq(s[3] - R(2) * s[2] + s[1]) + R(0.25) * (s[3] - s[1]) * (s[3] - s[1]);
  b[0] = k13 * sq(s[2] - R(2) * s[1] + s[0]) + R(0.25) * sq(R(3) * s[2] - R(4) * s[1] + s[0]);
  w_weights(b, 3, fabs(b[2] - b[0]), z);
  v[2] = R(11) * s[2] - R(7) * s[3] + R(2) * s[4];
  v[1] = -s[3] + R(5) * s[2] + R(2) * s[1];
  v[0] = R(2) * s[2] + R(5) * s[1] - s[0];
  sm = w5_blend(b, v);
}
// smoothness of the 4-point substencil (a, b, c, d) of WENO-7 with coefficient set K
template <class R, int K>
__device__ __forceinline__ R w7_beta(R a, R b, R c, R d) {
  constexpr double k[4][10] = {
    {2107.0, 9402.0, 7042.0, 1854.0, 11003.0, 17246.0, 4642.0, 7043.0, 3882.0, 547.0},
    {547.0, 2522.0, 1922.0, 494.0, 3443.0, 5966.0, 1602.0, 2843.0, 1642.0, 267.0},
    {267.0, 1642.0, 1602.0, 494.0, 2843.0, 5966.0, 1922.0, 3443.0, 2522.0, 547.0},
    {547.0, 3882.0, 4642.0, 1854.0, 7043.0, 17246.0, 7042.0, 11003.0, 9402.0, 2107.0}};
  return a * (R(k[K][0]) * a - R(k[K][1]) * b + R(k[K][2]) * c - R(k[K][3]) * d) +
         b * (R(k[K][4]) * b - R(k[K][5]) * c + R(k[K][6]) * d) + c * (R(k[K][7]) * c - R(k[K][8]) * d) +
         R(k[K][9]) * (d * d);
}
template <class R>
__device__ __forceinline__ R w7_blend(const R* b, const R* v) {
  const R a3 = R(1.0 / 35.0) * b[3], a2 = R(12.0 / 35.0) * b[2], a1 = R(18.0 / 35.0) * b[1],
          a0 = R(4.0 / 35.0) * b[0];
  const R ai = R(1) / (a3 + a2 + a1 + a0);
  return R(1.0 / 12.0) * ai * (a3 * v[3] + a2 * v[2] + a1 * v[1] + a0 * v[0]);
}
template <class R>
__device__ __forceinline__ void weno7z(const R* s, R& sm, R& sp) {
  R b[4], v[4];
  b[3] = w7_beta<R, 3>(s[0], s[1], s[2], s[3]);
  b[2] = w7_beta<R, 2>(s[1], s[2], s[3], s[4]);
  b[1] = w7_beta<R, 1>(s[2], s[3], s[4], s[5]);
  b[0] = w7_beta<R, 0>(s[3], s[4], s[5], s[6]);
  w_weights(b, 4, fabs(b[3] - b[0]), true);
  v[3] = R(-3) * s[0] + R(13) * s[1] - R(23) * s[2] + R(25) * s[3];
  v[2] = s[1] - R(5) * s[2] + R(13) * s[3] + R(3) * s[4];
  v[1] = -s[2] + R(7) * s[3] + R(7) * s[4] - s[5];
  v[0] = R(3) * s[3] + R(13) * s[4] - R(5) * s[5] + s[6];
  sp = w7_blend(b, v);
  b[3] = w7_beta<R, 3>(s[6], s[5], s[4], s[3]);
  b[2] = w7_beta<R, 2>(s[5], s[4], s[3], s[2]);
  b[1] = w7_beta<R, 1>(s[4], s[3], s[2], s[1]);
  b[0] = w7_beta<R, 0>(s[3], s[2], s[1], s[0]);
  w_weights(b, 4, fabs(b[3] - b[0]), true);
  v[3] = R(-3) * s[6] + R(13) * s[5] - R(23) * s[4] + R(25) * s[3];
  v[2] = s[5] - R(5) * s[4] + R(13) * s[3] + R(3) * s[2];
  v[1] = -s[4] + R(7) * s[3] + R(7) * s[2] - s[1];
  v[0] = R(3) * s[3] + R(13) * s[2] - R(5) * s[1] + s[0];
  sm = w7_blend(b, v);
}
template <class R>
__device__ __forceinline__ void weno3z(const R* s, R& sm, R& sp) {
  R b[2];
  b[1] = (s[0] - s[1]) * (s[0] - s[1]);
  b[0] = (s[1] - s[2]) * (s[1] - s[2]);
  w_weights(b, 2, fabs(b[1] - b[0]), true);
  R a1 = R(2) * b[1], a0 = R(1) * b[0], ai = R(1) / (a1 + a0);
  sp = R(0.5) * ai * (a1 * (-s[0] + R(3) * s[1]) + a0 * (s[1] + s[2]));
  b[1] = (s[2] - s[1]) * (s[2] - s[1]);
  b[0] = (s[1] - s[0]) * (s[1] - s[0]);
  w_weights(b, 2, fabs(b[1] - b[0]), true);
  a1 = R(2) * b[1];
  a0 = R(1) * b[0];
  ai = R(1) / (a1 + a0);
  sm = R(0.5) * ai * (a1 * (R(3) * s[1] - s[2]) + a0 * (s[0] + s[1]));
}
}  // namespace weno

// ------------------------------------------------------------------ PPM
// Source/PPM.H:28-115 (ppm_reconstruct)
template <class R>
__device__ __forceinline__ R vl_slope(R a, R b, R c) {
  // van Leer slope of Source/PPM.H:36-46 for the triple (a, b, c)
  const R dsl = R(2) * (b - a);
  const R dsr = R(2) * (c - b);
  R s = R(0);
  if (dsl * dsr > R(0)) {
    const R dsc = R(0.5) * (c - a);
    s = copysign(R(1), dsc) * dmin(fabs(dsc), dmin(fabs(dsl), fabs(dsr)));
  }
  return s;
}

// The interpolated value on the interface between a cell (value sl, van Leer slope dl)
// and its right neighbour (sr, dr), bounded by the two cell values (Source/PPM.H:61-65
// for sm, :93-97 for sp):
// the edge sm of the right cell is the edge sp of the left one, so a caller that holds
// the slopes of a row of cells forms each interface once.
template <class R>
__device__ __forceinline__ R ppm_edge(const R sl, const R sr, const R dl, const R dr) {
  R e = R(0.5) * (sr + sl) - (R(1) / R(6)) * (dr - dl);
  e = dmax(e, dmin(sr, sl));
  return dmin(e, dmax(sr, sl));
}

// Flattening and the monotonicity limiter of the parabola on the cell of value s2 with
// interface values sm, sp (Source/PPM.H:99-114).
template <class R>
__device__ __forceinline__ void ppm_limit(const R s2, const R flatn, R& sm, R& sp) {
  sm = flatn * sm + (R(1) - flatn) * s2;
  sp = flatn * sp + (R(1) - flatn) * s2;
  if ((sp - s2) * (s2 - sm) <= R(0)) {
    sp = s2;
    sm = s2;
  } else if (fabs(sp - s2) >= R(2) * fabs(sm - s2)) {
    sp = R(3) * s2 - R(2) * sm;
  } else if (fabs(sm - s2) >= R(2) * fabs(sp - s2)) {
    sm = R(3) * s2 - R(2) * sp;
  }
}

template <class R>
__device__ __forceinline__ void ppm_reconstruct(const R s0, const R s1, const R s2, const R s3, const R s4,
                                                const R flatn, R& sm, R& sp) {
  const R d1 = vl_slope(s0, s1, s2), d2 = vl_slope(s1, s2, s3), d3 = vl_slope(s2, s3, s4);
  sm = ppm_edge(s1, s2, d1, d2);
  sp = ppm_edge(s2, s3, d2, d3);
  ppm_limit(s2, flatn, sm, sp);
}

// Source/PPM.H:131-189 (ppm_int_profile), one wave
template <class R>
__device__ __forceinline__ void ppm_wave(R sm, R sp, R s6, R speed, R dtdx, R& Ip, R& Im) {
  const R sigma = fabs(speed) * dtdx;
  if (speed <= R(0)) {
    Ip = sp;
    Im = sm + R(0.5) * sigma * (sp - sm + (R(1) - (R(2) / R(3)) * sigma) * s6);
  } else {
    Ip = sp - R(0.5) * sigma * (sp - sm - (R(1) - (R(2) / R(3)) * sigma) * s6);
    Im = sm;
  }
}

template <class R>
__device__ __forceinline__ R ppm_s6(R sm, R sp, R sc) { return R(6) * sc - R(3) * (sm + sp); }

// Source/Godunov.H:188-260 (flatten); the stencil +-3 lies inside the q FAB for every
// cell the path traces (the q FAB covers grow(box,4), traced cells grow(box,1)). q is any
// accessor q(i, j, k, qcomp) of the primitive state.
template <class R, class Q>
__device__ __forceinline__ R flatten(const Q& q, int i, int j, int k, int dir) {
  const int di = dir == 0, dj = dir == 1, dk = dir == 2;
#define QS(s, n) R(q(i + (s) * di, j + (s) * dj, k + (s) * dk, n))
  const int n = pcg::QPRES;
  const R small_pres = Lim<R>::small_pres();
  const R shktst = R(0.33e0);
  const R zcut1 = R(0.75e0);
  const R zcut2 = R(0.85e0);
  const R dzcut = R(1) / (zcut2 - zcut1);
  const R qm = QS(-1, n);
  const R qp = QS(1, n);
  const R qmun = QS(-1, pcg::QU + dir);
  const R qpun = QS(1, pcg::QU + dir);
  const R qmm = QS(-2, n);
  const R qpp = QS(2, n);
  R dp = qp - qm;
  const int ishft = (dp > R(0)) ? 1 : -1;
  R denom = dmax(small_pres, fabs(qpp - qmm));
  R zeta = fabs(dp) / denom;
  const R z = min1_max0<R>(dzcut * (zeta - zcut1));
  R tst = (qmun - qpun >= R(0)) ? R(1) : R(0);
  R tmp = dmin(qp, qm);
  const R chi = (fabs(dp) / tmp) > shktst ? tst : R(0);
  const R qpshft = QS(1 - ishft, n);
  const R qmshft = QS(-(1 + ishft), n);
  const R qpunshft = QS(1 - ishft, pcg::QU + dir);
  const R qmunshft = QS(-(1 + ishft), pcg::QU + dir);
  const R qppshft = QS(2 - ishft, n);
  const R qmmshft = QS(-(2 + ishft), n);
  dp = qpshft - qmshft;
  denom = dmax(small_pres, fabs(qppshft - qmmshft));
  zeta = fabs(dp) / denom;
  const R z2 = min1_max0<R>(dzcut * (zeta - zcut1));
  tst = (qmunshft - qpunshft >= R(0)) ? R(1) : R(0);
  tmp = dmin(qpshft, qmshft);
  const R chi2 = (fabs(dp) / tmp) > shktst ? tst : R(0);
  return R(1) - dmax(chi2 * z2, chi * z);
#undef QS
}

// Source/PLM.H:21-77 (plm_slope)
template <class R>
__device__ __forceinline__ R plm_slope(R qm2, R qm, R qc, R qp, R qp2, R flat, int order) {
  if (order == 1) return R(0);
  R dlft, drgt, dcen, dfm = R(0), dfp = R(0), dlim, dsgn, dtemp;
  if (order == 4) {
    dlft = qm - qm2;
    drgt = qc - qm;
    dcen = R(0.5) * (dlft + drgt);
    dsgn = copysign(R(1), dcen);
    dlim = (dlft * drgt >= R(0)) ? R(2) * dmin(fabs(dlft), fabs(drgt)) : R(0);
    dfm = dsgn * dmin(dlim, fabs(dcen));
    dlft = qp - qc;
    drgt = qp2 - qp;
    dcen = R(0.5) * (dlft + drgt);
    dsgn = copysign(R(1), dcen);
    dlim = (dlft * drgt >= R(0)) ? R(2) * dmin(fabs(dlft), fabs(drgt)) : R(0);
    dfp = dsgn * dmin(dlim, fabs(dcen));
  }
  dlft = qc - qm;
  drgt = qp - qc;
  dcen = R(0.5) * (dlft + drgt);
  dsgn = copysign(R(1), dcen);
  dlim = (dlft * drgt >= R(0)) ? R(2) * dmin(fabs(dlft), fabs(drgt)) : R(0);
  dtemp = (order == 2) ? dcen : R(4) / R(3) * dcen - R(1) / R(6) * (dfp + dfm);
  return flat * dsgn * dmin(dlim, fabs(dtemp));
}

// ------------------------------------------------------------------ Riemann
template <int NS, class R>
struct FaceState {
  R rho, un, ut1, ut2, p;
  R y[NS];
};

template <class R>
struct RiemannOut {
  R ustar, frho, fun, fut1, fut2, feden, feint, gun, gpres;
  R gut1, gut2, regd;  // the Godunov state's tangential velocities and rho*e (qint)
};

// Source/Riemann.H:9-200 (riemann), omega = rad = 0, bc_test_val = 1. The EOS calls
// whose results the reference overwrites unused (RYP2E at :94, :111, :153) are not
// evaluated; they do not affect any output.
// Source/Riemann.H:9-200 in the reduced algebra of the FMA/mixed forms (see EosR):
// the same states, masks and blends, with the species normalisations folded into one
// reciprocal per state and rho*e of the Godunov state taken directly as
// sum(rho Y_k e_k(T)).
template <int NS, bool MIX, class R>
__device__ __forceinline__ void riemann_reduced(const FaceState<NS, R>& L, const FaceState<NS, R>& Rs, R cav,
                                                R p0, RiemannOut<R>& o) {
  using ER = EosR<NS, MIX, R>;
  const R rl = L.rho, ul = L.un, vl = L.ut1, v2l = L.ut2, pl = L.p;
  const R rr = Rs.rho, ur = Rs.un, vr = Rs.ut1, v2r = Rs.ut2, pr = Rs.p;
  const R wsmall = Lim<R>::tiny();
  const R cl = ER::cs_y(rl, pabs(pl, p0), L.y);
  const R cr = ER::cs_y(rr, pabs(pr, p0), Rs.y);
  const R wl = dmax(wsmall, cl * rl);
  const R wr = dmax(wsmall, cr * rr);
  const R iwlr = rrcp(wl + wr);
  // the star state as the left state plus weighted jumps: (wr pl + wl pr + wl wr (ul - ur))
  // / (wl + wr) and (wl ul + wr ur + pl - pr) / (wl + wr) rearranged, so that equal left and
  // right pressures (velocities) give exactly that pressure (velocity) without FP32
  // rounding noise in uniform regions
  const R pstar = dmax(pfloor(Lim<R>::tiny(), p0), pl + (wl * (pr - pl) + wl * wr * (ul - ur)) * iwlr);
  R ustar = ul + (wr * (ur - ul) + (pl - pr)) * iwlr;
  bool mask = ustar > R(0);
  R uo = mask ? ul : ur;
  R po = mask ? pl : pr;
  const bool mid = fabs(ustar) < R(pcg::SMALLU) * R(0.5) * (fabs(ul) + fabs(ur)) || ustar == R(0);
  ustar = mid ? R(0) : ustar;
  uo = mid ? R(0.5) * (ul + ur) : uo;
  po = mid ? R(0.5) * (pl + pr) : po;
  R rspo[NS];
  R ro = R(0);
  if constexpr (sizeof(R) == 4 && NS > 1) {
    // the upwind (or averaged) partial densities as al * yL + ar * yR, species in pairs
    const R al = mid ? R(0.5) * rl : (mask ? rl : R(0));
    const R ar = mid ? R(0.5) * rr : (mask ? R(0) : rr);
    ro = blend2_sum<NS>(al, L.y, ar, Rs.y, rspo);
  } else {
#pragma unroll
    for (int n = 0; n < NS; n++) {
      rspo[n] = mid ? R(0.5) * (rl * L.y[n] + rr * Rs.y[n]) : (mask ? rl * L.y[n] : rr * Rs.y[n]);
      ro += rspo[n];
    }
  }
  const R co = ER::cs_w(ro, pabs(po, p0), rspo);
  const R drho = rdiv(pstar - po, co * co);
  const R gscale = R(1) + drho * rrcp(ro);
  R rspstar[NS];
  R rstar = R(0);
#pragma unroll
  for (int n = 0; n < NS; n++) {
    rspstar[n] = dmax(R(0), rspo[n] * gscale);
    rstar += rspstar[n];
  }
  const R cstar = ER::cs_w(rstar, pabs(pstar, p0), rspstar);
  const R sgnm = copysign(R(1), ustar);
  R spout = co - sgnm * uo;
  R spin = cstar - sgnm * ustar;
  const R ushock = R(0.5) * (spin + spout);
  mask = pstar < po;
  spout = mask ? spout : ushock;
  spin = mask ? spin : ushock;
  const R scr = (fabs(spout - spin) < Lim<R>::very_small()) ? R(pcg::SMALL_NUM) * cav : spout - spin;
  const R frac = max0_min1<R>((R(1) + rdiv(spout + spin, scr)) * R(0.5));
  mask = ustar > R(0);
  R qint_iv1 = mask ? vl : vr;
  R qint_iv2 = mask ? v2l : v2r;
  mask = (ustar == R(0));
  qint_iv1 = mask ? R(0.5) * (vl + vr) : qint_iv1;
  qint_iv2 = mask ? R(0.5) * (v2l + v2r) : qint_iv2;
  // final Godunov state: star (spin >= 0), original (spout < 0) or the fan blend
  const bool use_star = spin >= R(0);
  const bool use_orig = !use_star && (spout < R(0));
  const R qint_iu = use_star ? ustar : use_orig ? uo : frac * ustar + (R(1) - frac) * uo;
  const R qint_gdpres = use_star ? pstar : use_orig ? po : frac * pstar + (R(1) - frac) * po;
  R rgd = R(0);
  if constexpr (sizeof(R) == 4 && NS > 1) {
    const R cs = use_star ? R(1) : use_orig ? R(0) : frac;
    const R cn = use_star ? R(0) : use_orig ? R(1) : R(1) - frac;
    rgd = blend2_sum<NS>(cs, rspstar, cn, rspo, rspo);
  } else {
#pragma unroll
    for (int n = 0; n < NS; n++) {
      rspo[n] = use_star ? rspstar[n] : use_orig ? rspo[n] : frac * rspstar[n] + (R(1) - frac) * rspo[n];
      rgd += rspo[n];
    }
  }
  const R regd = ER::rhoe_w(pabs(qint_gdpres, p0), rspo);
  const R frho = rgd * qint_iu;
  o.ustar = ustar;
  o.frho = frho;
  o.fun = frho * qint_iu + qint_gdpres;
  o.fut1 = frho * qint_iv1;
  o.fut2 = frho * qint_iv2;
  const R rhoetot = regd + R(0.5) * rgd * (qint_iu * qint_iu + qint_iv1 * qint_iv1 + qint_iv2 * qint_iv2);
  o.feden = qint_iu * (rhoetot + pabs(qint_gdpres, p0));
  o.feint = qint_iu * regd;
  o.gun = qint_iu;
  o.gpres = qint_gdpres;
  o.gut1 = qint_iv1;
  o.gut2 = qint_iv2;
  o.regd = regd;
}

template <int NS, bool MIX, class R>
__device__ __forceinline__ void riemann(const FaceState<NS, R>& L, const FaceState<NS, R>& Rs, R cav,
                                        RiemannOut<R>& o) {
  using E = Eos<NS, MIX, R>;
  const R rl = L.rho, ul = L.un, vl = L.ut1, v2l = L.ut2, pl = L.p;
  const R rr = Rs.rho, ur = Rs.un, vr = Rs.ut1, v2r = Rs.ut2, pr = Rs.p;
  const R wsmall = Lim<R>::tiny();
  const R cl = E::rpy2cs(rl, pl, L.y);
  const R cr = E::rpy2cs(rr, pr, Rs.y);
  const R wl = dmax(wsmall, cl * rl);
  const R wr = dmax(wsmall, cr * rr);
  const R pstar = dmax(Lim<R>::tiny(), ((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr));
  R ustar = ((wl * ul + wr * ur) + (pl - pr)) / (wl + wr);

  bool mask = ustar > R(0);
  R rspo[NS];
  R ro = R(0);
#pragma unroll
  for (int n = 0; n < NS; n++) {
    rspo[n] = mask ? rl * L.y[n] : rr * Rs.y[n];
    ro += rspo[n];
  }
  R uo = mask ? ul : ur;
  R po = mask ? pl : pr;
  mask = fabs(ustar) < R(pcg::SMALLU) * R(0.5) * (fabs(ul) + fabs(ur)) || ustar == R(0);
  ustar = mask ? R(0) : ustar;
  ro = R(0);
#pragma unroll
  for (int n = 0; n < NS; n++) {
    rspo[n] = mask ? R(0.5) * (rl * L.y[n] + rr * Rs.y[n]) : rspo[n];
    ro += rspo[n];
  }
  uo = mask ? R(0.5) * (ul + ur) : uo;
  po = mask ? R(0.5) * (pl + pr) : po;

  R ytmp[NS];
#pragma unroll
  for (int n = 0; n < NS; n++) ytmp[n] = rspo[n] / ro;
  const R co = E::rpy2cs(ro, po, ytmp);

  const R drho = (pstar - po) / (co * co);
  R rspstar[NS];
  R rstar = R(0);
#pragma unroll
  for (int n = 0; n < NS; n++) {
    const R spon = rspo[n] / ro;
    rspstar[n] = dmax(R(0), rspo[n] + drho * spon);
    rstar += rspstar[n];
  }
#pragma unroll
  for (int n = 0; n < NS; n++) ytmp[n] = rspstar[n] / rstar;
  const R cstar = E::rpy2cs(rstar, pstar, ytmp);

  const R sgnm = copysign(R(1), ustar);
  R spout = co - sgnm * uo;
  R spin = cstar - sgnm * ustar;
  const R ushock = R(0.5) * (spin + spout);
  mask = pstar < po;
  spout = mask ? spout : ushock;
  spin = mask ? spin : ushock;
  const R scr = (fabs(spout - spin) < Lim<R>::very_small()) ? R(pcg::SMALL_NUM) * cav : spout - spin;
  const R frac = max0_min1<R>((R(1) + (spout + spin) / scr) * R(0.5));

  mask = ustar > R(0);
  R qint_iv1 = mask ? vl : vr;
  R qint_iv2 = mask ? v2l : v2r;
  mask = (ustar == R(0));
  qint_iv1 = mask ? R(0.5) * (vl + vr) : qint_iv1;
  qint_iv2 = mask ? R(0.5) * (v2l + v2r) : qint_iv2;
  R rspgd[NS];
#pragma unroll
  for (int n = 0; n < NS; n++) rspgd[n] = frac * rspstar[n] + (R(1) - frac) * rspo[n];
  R qint_iu = frac * ustar + (R(1) - frac) * uo;
  R qint_gdpres = frac * pstar + (R(1) - frac) * po;

  mask = (spout < R(0));
#pragma unroll
  for (int n = 0; n < NS; n++) rspgd[n] = mask ? rspo[n] : rspgd[n];
  qint_iu = mask ? uo : qint_iu;
  qint_gdpres = mask ? po : qint_gdpres;
  mask = (spin >= R(0));
  R rgd = R(0);
#pragma unroll
  for (int n = 0; n < NS; n++) {
    rspgd[n] = mask ? rspstar[n] : rspgd[n];
    rgd += rspgd[n];
  }
  qint_iu = mask ? ustar : qint_iu;
  qint_gdpres = mask ? pstar : qint_gdpres;

#pragma unroll
  for (int n = 0; n < NS; n++) ytmp[n] = rspgd[n] / rgd;
  const R gdnv_e = E::ryp2e(rgd, ytmp, qint_gdpres);
  const R regd = rgd * gdnv_e;

  const R frho = rgd * qint_iu;
  o.ustar = ustar;
  o.frho = frho;
  o.fun = frho * qint_iu + qint_gdpres;
  o.fut1 = frho * qint_iv1;
  o.fut2 = frho * qint_iv2;
  const R rhoetot = regd + R(0.5) * rgd * (qint_iu * qint_iu + qint_iv1 * qint_iv1 + qint_iv2 * qint_iv2);
  o.feden = qint_iu * (rhoetot + qint_gdpres);
  o.feint = qint_iu * regd;
  o.gun = qint_iu;
  o.gpres = qint_gdpres;
  o.gut1 = qint_iv1;
  o.gut2 = qint_iv2;
  o.regd = regd;
}

// Source/Godunov.H:303-449 (pc_cmpflx): boundary overrides at the domain faces
// (:378-418), the Riemann solve, and the upwinded species fluxes (:15-25, :438-441).
// The face states are in absolute velocity order (u, v, w); fl[] receives URHO, UMX,
// UMY, UMZ, UEDEN, UEINT and the species fluxes in absolute order. DIR is the normal.
// With QX, qx[0..2] also receive the Godunov state's tangential velocities (t1, t2 in
// absolute order) and rho*e, from which pc_umeth_3D's qint GDGAME is formed.
template <int NS, bool MIX, bool EXACT, int DIR, class R, bool QX = false>
__device__ __forceinline__ void cmpflx(const R* ql, const R* qr, int idx, int bclo, int bchi, int domlo, int domhi,
                                       R cav, R p0, R* fl, R& gun, R& gpres, R* qx = nullptr) {
  constexpr int t1 = (DIR == 0) ? 1 : 0;
  constexpr int t2 = (DIR == 2) ? 1 : 2;
  FaceState<NS, R> L, Rs;
  L.rho = ql[pcg::TR_RHO];
  L.un = ql[pcg::TR_U + DIR];
  L.ut1 = ql[pcg::TR_U + t1];
  L.ut2 = ql[pcg::TR_U + t2];
  L.p = ql[pcg::TR_P];
  Rs.rho = qr[pcg::TR_RHO];
  Rs.un = qr[pcg::TR_U + DIR];
  Rs.ut1 = qr[pcg::TR_U + t1];
  Rs.ut2 = qr[pcg::TR_U + t2];
  Rs.p = qr[pcg::TR_P];
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    L.y[n] = ql[pcg::TR_Y + n];
    Rs.y[n] = qr[pcg::TR_Y + n];
  }
  if (idx == domlo) {
    if (bclo == pcg::BC_NO_SLIP_WALL || bclo == pcg::BC_SLIP_WALL || bclo == pcg::BC_SYMMETRY) {
      L.un = -Rs.un; L.ut1 = Rs.ut1; L.ut2 = Rs.ut2; L.p = Rs.p; L.rho = Rs.rho;
    } else if (bclo == pcg::BC_OUTFLOW) {
      L.un = Rs.un; L.ut1 = Rs.ut1; L.ut2 = Rs.ut2; L.p = Rs.p; L.rho = Rs.rho;
    }
  } else if (idx == domhi + 1) {
    if (bchi == pcg::BC_NO_SLIP_WALL || bchi == pcg::BC_SLIP_WALL || bchi == pcg::BC_SYMMETRY) {
      Rs.un = -L.un; Rs.ut1 = L.ut1; Rs.ut2 = L.ut2; Rs.p = L.p; Rs.rho = L.rho;
    } else if (bchi == pcg::BC_OUTFLOW) {
      Rs.un = L.un; Rs.ut1 = L.ut1; Rs.ut2 = L.ut2; Rs.p = L.p; Rs.rho = L.rho;
    }
  }
  RiemannOut<R> o;
  if (EXACT)
    riemann<NS, MIX, R>(L, Rs, cav, o);
  else
    riemann_reduced<NS, MIX, R>(L, Rs, cav, p0, o);
  fl[pcg::URHO] = o.frho;
  fl[pcg::UMX + DIR] = o.fun;
  fl[pcg::UMX + t1] = o.fut1;
  fl[pcg::UMX + t2] = o.fut2;
  fl[pcg::UEDEN] = o.feden;
  fl[pcg::UEINT] = o.feint;
  const R flxrho = o.frho;
  if constexpr (sizeof(R) == 4 && NS > 1) {
    // pc_cmpflx_passive as ca * yL + cb * yR, species in pairs
    const R ca = (o.ustar > R(0)) ? flxrho : (o.ustar < R(0)) ? R(0) : flxrho * R(0.5);
    const R cb = (o.ustar > R(0)) ? R(0) : (o.ustar < R(0)) ? flxrho : flxrho * R(0.5);
    blend2_sum<NS>(ca, ql + pcg::TR_Y, cb, qr + pcg::TR_Y, fl + pcg::UFS);
  } else {
#pragma unroll
    for (int n = 0; n < NS; n++) {
      const R a = ql[pcg::TR_Y + n], b = qr[pcg::TR_Y + n];
      fl[pcg::UFS + n] = (o.ustar > R(0)) ? flxrho * a : (o.ustar < R(0)) ? flxrho * b : flxrho * R(0.5) * (a + b);
    }
  }
  gun = o.gun;
  gpres = o.gpres;
  if constexpr (QX) {
    qx[0] = o.gut1;
    qx[1] = o.gut2;
    qx[2] = o.regd;
  }
}

}  // namespace PCG_TU
