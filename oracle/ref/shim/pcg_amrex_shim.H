// pcg_amrex_shim.H -- the small subset of the AMReX API that the reference's Godunov
// hot-path sources use, so that those sources compile unmodified, in place, as a CPU
// FP64 library (test infrastructure: the oracle/_ref build). Written from the AMReX
// interface as the reference calls it; nothing here is AMReX code.
//
// Semantics that matter for results:
//  * Array4 addressing p[(i-b.x) + (j-b.y)*js + (k-b.z)*ks + n*ns], end exclusive;
//    contains() tests [begin, end).
//  * Box keeps a per-direction node flag so surroundingNodes/enclosedCells round-trip.
//  * ParallelFor visits every cell of the box (order irrelevant: the reference kernels
//    write disjoint cells).
//  * amrex::min/max are std::min/std::max.
#ifndef PCG_AMREX_SHIM_H
#define PCG_AMREX_SHIM_H

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <limits>
#include <string>
#include <type_traits>
#include <vector>

#define AMREX_SPACEDIM 3
#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST
#define AMREX_GPU_HOST_DEVICE
#define AMREX_FORCE_INLINE inline
#define AMREX_INLINE inline
#define AMREX_D_DECL(a, b, c) a, b, c
#define AMREX_D_TERM(a, b, c) a b c
#define AMREX_D_PICK(a, b, c) c
#define BL_PROFILE(x)
#define BL_PROFILE_VAR(x, y)
#define AMREX_ASSERT(x)
#define AMREX_ALWAYS_ASSERT(x)
#define AMREX_ALWAYS_ASSERT_WITH_MESSAGE(x, m)

namespace amrex {

using Real = double;

template <class T>
constexpr const T& min(const T& a, const T& b) noexcept { return std::min(a, b); }
template <class T>
constexpr const T& max(const T& a, const T& b) noexcept { return std::max(a, b); }

namespace Math {
using std::abs;
using std::copysign;
template <class T>
constexpr T pi() { return T(3.1415926535897932384626433832795029L); }
} // namespace Math

template <class... Ts>
inline void ignore_unused(const Ts&...) {}

[[noreturn]] inline void Error(const char* msg) {
  std::fprintf(stderr, "amrex::Error: %s\n", msg);
  std::abort();
}
[[noreturn]] inline void Abort(const char* msg) { Error(msg); }
inline void Error(const std::string& msg) { Error(msg.c_str()); }
inline void Abort(const std::string& msg) { Error(msg.c_str()); }

template <class T, unsigned int N>
struct GpuArray {
  T arr[N];
  T& operator[](int i) noexcept { return arr[i]; }
  const T& operator[](int i) const noexcept { return arr[i]; }
  T* data() noexcept { return arr; }
  const T* data() const noexcept { return arr; }
  static constexpr unsigned int size() { return N; }
};

template <class T>
using Vector = std::vector<T>;

struct Dim3 {
  int x, y, z;
};

struct IntVect {
  int v[3];
  IntVect() : v{0, 0, 0} {}
  explicit IntVect(int a) : v{a, a, a} {}
  IntVect(int a, int b, int c) : v{a, b, c} {}
  int& operator[](int d) { return v[d]; }
  const int& operator[](int d) const { return v[d]; }
  static IntVect TheDimensionVector(int d) { return IntVect(d == 0, d == 1, d == 2); }
  static IntVect TheZeroVector() { return IntVect(0); }
  static IntVect TheUnitVector() { return IntVect(1); }
  IntVect operator+(const IntVect& o) const { return IntVect(v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]); }
  IntVect operator-(const IntVect& o) const { return IntVect(v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]); }
  IntVect operator-() const { return IntVect(-v[0], -v[1], -v[2]); }
  IntVect& operator+=(const IntVect& o) { for (int d = 0; d < 3; ++d) v[d] += o.v[d]; return *this; }
  IntVect& operator-=(const IntVect& o) { for (int d = 0; d < 3; ++d) v[d] -= o.v[d]; return *this; }
  bool operator==(const IntVect& o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
};
inline IntVect operator*(int s, const IntVect& a) { return IntVect(s * a.v[0], s * a.v[1], s * a.v[2]); }
inline IntVect operator*(const IntVect& a, int s) { return s * a; }

struct RealVect {
  Real v[3];
  RealVect() : v{0, 0, 0} {}
  RealVect(Real a, Real b, Real c) : v{a, b, c} {}
  Real& operator[](int d) { return v[d]; }
  const Real& operator[](int d) const { return v[d]; }
  RealVect operator-(const RealVect& o) const { return RealVect(v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]); }
  Real radSquared() const { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; }
};

struct Box {
  IntVect lo, hi;
  int node[3] = {0, 0, 0};
  Box() : lo(0), hi(-1) {}
  Box(const IntVect& l, const IntVect& h) : lo(l), hi(h) {}
  const IntVect& smallEnd() const { return lo; }
  const IntVect& bigEnd() const { return hi; }
  int smallEnd(int d) const { return lo[d]; }
  int bigEnd(int d) const { return hi[d]; }
  GpuArray<int, 3> loVect3d() const { return {{lo[0], lo[1], lo[2]}}; }
  GpuArray<int, 3> hiVect3d() const { return {{hi[0], hi[1], hi[2]}}; }
  const int* loVect() const { return lo.v; }
  const int* hiVect() const { return hi.v; }
  bool ok() const { return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2]; }
  Box& grow(int n) { for (int d = 0; d < 3; ++d) { lo[d] -= n; hi[d] += n; } return *this; }
  Box& grow(int d, int n) { lo[d] -= n; hi[d] += n; return *this; }
  Box& growHi(int d, int n) { hi[d] += n; return *this; }
  Box& growLo(int d, int n) { lo[d] -= n; return *this; }
  Box& setBig(int d, int v) { hi[d] = v; return *this; }
  Box& setSmall(int d, int v) { lo[d] = v; return *this; }
  long numPts() const { return ok() ? long(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1) : 0; }
  bool contains(const IntVect& p) const {
    return p[0] >= lo[0] && p[0] <= hi[0] && p[1] >= lo[1] && p[1] <= hi[1] && p[2] >= lo[2] && p[2] <= hi[2];
  }
  static Box TheUnitBox() { return Box(IntVect(0), IntVect(0)); }
};
inline Box grow(Box b, int n) { return b.grow(n); }
inline Box grow(Box b, int d, int n) { return b.grow(d, n); }
inline Box grow(Box b, const IntVect& n) { for (int d = 0; d < 3; ++d) b.grow(d, n[d]); return b; }
inline Box growHi(Box b, int d, int n) { return b.growHi(d, n); }
inline Box growLo(Box b, int d, int n) { return b.growLo(d, n); }
inline Box surroundingNodes(Box b, int d) {
  if (!b.node[d]) { b.hi[d] += 1; b.node[d] = 1; }
  return b;
}
inline Box surroundingNodes(Box b) { for (int d = 0; d < 3; ++d) b = surroundingNodes(b, d); return b; }
inline Box enclosedCells(Box b, int d) {
  if (b.node[d]) { b.hi[d] -= 1; b.node[d] = 0; }
  return b;
}
inline Box enclosedCells(Box b) { for (int d = 0; d < 3; ++d) b = enclosedCells(b, d); return b; }
inline Box operator&(const Box& a, const Box& b) {
  Box r;
  for (int d = 0; d < 3; ++d) { r.lo[d] = std::max(a.lo[d], b.lo[d]); r.hi[d] = std::min(a.hi[d], b.hi[d]); }
  return r;
}

template <class T>
struct Array4 {
  T* p = nullptr;
  long jstride = 0, kstride = 0, nstride = 0;
  Dim3 begin{0, 0, 0}, end{0, 0, 0};
  int ncomp = 0;

  Array4() = default;
  Array4(T* ptr, Dim3 b, Dim3 e, int nc)
    : p(ptr), jstride(e.x - b.x), kstride(long(e.x - b.x) * (e.y - b.y)),
      nstride(long(e.x - b.x) * (e.y - b.y) * (e.z - b.z)), begin(b), end(e), ncomp(nc) {}
  Array4(T* ptr, long js, long ks, long ns, Dim3 b, Dim3 e, int nc)
    : p(ptr), jstride(js), kstride(ks), nstride(ns), begin(b), end(e), ncomp(nc) {}
  template <class U, class = std::enable_if_t<std::is_same<const U, T>::value && !std::is_same<U, T>::value>>
  Array4(const Array4<U>& o)
    : p(o.p), jstride(o.jstride), kstride(o.kstride), nstride(o.nstride), begin(o.begin), end(o.end),
      ncomp(o.ncomp) {}

  T& operator()(int i, int j, int k) const {
    return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride];
  }
  T& operator()(int i, int j, int k, int n) const {
    return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride];
  }
  T& operator()(const IntVect& iv) const { return (*this)(iv[0], iv[1], iv[2]); }
  T& operator()(const IntVect& iv, int n) const { return (*this)(iv[0], iv[1], iv[2], n); }
  bool contains(int i, int j, int k) const {
    return i >= begin.x && i < end.x && j >= begin.y && j < end.y && k >= begin.z && k < end.z;
  }
  int nComp() const { return ncomp; }
  T* dataPtr() const { return p; }
  explicit operator bool() const { return p != nullptr; }
};

struct Arena {};
inline Arena* The_Async_Arena() { return nullptr; }
inline Arena* The_Arena() { return nullptr; }

enum class RunOn { Host, Device, Gpu = Device, Cpu = Host };

template <class T>
struct BaseFab {
  Box box;
  int nc = 0;
  std::vector<T> data;
  BaseFab() = default;
  BaseFab(const Box& b, int n, Arena* = nullptr) { resize(b, n); }
  void resize(const Box& b, int n, Arena* = nullptr) {
    box = b;
    nc = n;
    data.assign(size_t(b.numPts()) * size_t(n), T(0));
  }
  Array4<T> array() {
    return Array4<T>(data.data(), Dim3{box.lo[0], box.lo[1], box.lo[2]},
                     Dim3{box.hi[0] + 1, box.hi[1] + 1, box.hi[2] + 1}, nc);
  }
  Array4<const T> array() const { return const_array(); }
  Array4<const T> const_array() const {
    return Array4<const T>(data.data(), Dim3{box.lo[0], box.lo[1], box.lo[2]},
                           Dim3{box.hi[0] + 1, box.hi[1] + 1, box.hi[2] + 1}, nc);
  }
  template <RunOn R = RunOn::Host>
  void setVal(T v) { std::fill(data.begin(), data.end(), v); }
  int nComp() const { return nc; }
  const Box& box_() const { return box; }
};
using FArrayBox = BaseFab<Real>;
using IArrayBox = BaseFab<int>;

template <class F>
inline void ParallelFor(const Box& b, F&& f) {
  for (int k = b.lo[2]; k <= b.hi[2]; ++k)
    for (int j = b.lo[1]; j <= b.hi[1]; ++j)
      for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k);
}
template <class F>
inline void ParallelFor(const Box& b, int ncomp, F&& f) {
  for (int n = 0; n < ncomp; ++n)
    for (int k = b.lo[2]; k <= b.hi[2]; ++k)
      for (int j = b.lo[1]; j <= b.hi[1]; ++j)
        for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k, n);
}
template <class F>
inline void Loop(const Box& b, F&& f) { ParallelFor(b, std::forward<F>(f)); }

// Embedded-boundary cell flag: every cell is regular in this build (the EB halves of
// the reference files only need to compile).
struct EBCellFlag {
  bool isCovered() const { return false; }
  bool isRegular() const { return true; }
  bool isSingleValued() const { return false; }
  bool isMultiValued() const { return false; }
  bool isConnected(int, int, int) const { return true; }
  bool isConnected(const IntVect&) const { return true; }
  int numNeighbors() const { return 26; }
};

namespace PhysBCType {
enum physicalBndryTypes { interior = 0, inflow, outflow, symmetry, slipwall, noslipwall };
}

struct GeometryData {
  Real prob_lo[3] = {0, 0, 0};
  Real dx[3] = {1, 1, 1};
  Real ProbLo(int d) const { return prob_lo[d]; }
  Real CellSize(int d) const { return dx[d]; }
};
class Geometry;
class MFIter;
class EBFArrayBoxFactory;
struct BCRec {};

namespace Gpu {
inline void synchronize() {}
} // namespace Gpu

} // namespace amrex

#endif
