/* Minimal stand-in for the AMReX types the reference transfer operators and
 * boundary conditions use (Box with its index type, IntVect, FArrayBox,
 * Geometry, ParallelFor and the Interpolater base class).
 * Semantics follow AMReX: boxes are inclusive [lo, hi]; FArrayBox data is
 * Fortran ordered (x fastest) with component stride numPts(); coarsen uses
 * floor division.  Oracle build only. */
#ifndef CX_REF_STUB_AMREX_INTERPOLATER_H
#define CX_REF_STUB_AMREX_INTERPOLATER_H
#include <cstddef>
#include <vector>

namespace amrex {
typedef double Real;
template <typename T> using Vector = std::vector<T>;
enum class RunOn { Gpu, Cpu, Device = Gpu, Host = Cpu };

struct IntVect {
  int v[3];
  IntVect() : v{0, 0, 0} {}
  explicit IntVect(int a) : v{a, a, a} {}
  IntVect(int a, int b, int c) : v{a, b, c} {}
  const int *getVect() const { return v; }
  int operator[](int d) const { return v[d]; }
  int &operator[](int d) { return v[d]; }
  bool operator==(const IntVect &o) const {
    return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2];
  }
};

inline int cx_floordiv(int a, int b) {
  return a >= 0 ? a / b : -((-a + b - 1) / b);
}

struct IndexType {
  enum CellIndex { CELL = 0, NODE = 1 };
};

struct Box {
  IntVect lo, hi;
  IndexType::CellIndex typ[3] = {IndexType::CELL, IndexType::CELL, IndexType::CELL};
  Box() {}
  Box(const IntVect &l, const IntVect &h) : lo(l), hi(h) {}
  const int *loVect() const { return lo.v; }
  const int *hiVect() const { return hi.v; }
  const IntVect &smallEnd() const { return lo; }
  const IntVect &bigEnd() const { return hi; }
  int smallEnd(int d) const { return lo[d]; }
  int bigEnd(int d) const { return hi[d]; }
  IndexType::CellIndex type(int d) const { return typ[d]; }
  bool ok() const { return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2]; }
  long numPts() const {
    return ok() ? long(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) *
                      (hi[2] - lo[2] + 1)
                : 0;
  }
  long index(const IntVect &p) const {
    const long nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1;
    return (p[0] - lo[0]) + nx * ((p[1] - lo[1]) + ny * long(p[2] - lo[2]));
  }
  bool contains(const IntVect &p) const {
    for (int d = 0; d < 3; ++d)
      if (p[d] < lo[d] || p[d] > hi[d])
        return false;
    return true;
  }
  Box &grow(int d, int n) {
    lo[d] -= n;
    hi[d] += n;
    return *this;
  }
  Box operator&(const Box &o) const {
    Box r;
    for (int d = 0; d < 3; ++d) {
      r.lo[d] = lo[d] > o.lo[d] ? lo[d] : o.lo[d];
      r.hi[d] = hi[d] < o.hi[d] ? hi[d] : o.hi[d];
    }
    return r;
  }
  bool operator==(const Box &o) const { return lo == o.lo && hi == o.hi; }
};

inline Box coarsen(const Box &b, int r) {
  Box c;
  for (int d = 0; d < 3; ++d) {
    c.lo[d] = cx_floordiv(b.lo[d], r);
    c.hi[d] = cx_floordiv(b.hi[d], r);
  }
  return c;
}

struct FArrayBox {
  Box bx;
  double *ptr;
  int ncomp;
  FArrayBox(const Box &b, double *p, int n) : bx(b), ptr(p), ncomp(n) {}
  const Box &box() const { return bx; }
  const double *dataPtr(int c = 0) const { return ptr + c * bx.numPts(); }
  double *dataPtr(int c = 0) { return ptr + c * bx.numPts(); }
  int nComp() const { return ncomp; }
};
struct IArrayBox {};
// The level's cell-centred domain box and its physical extent.
struct Geometry {
  Box domain;
  double problo[3] = {0, 0, 0}, probhi[3] = {1, 1, 1}, dx[3] = {1, 1, 1};
  const Box &Domain() const { return domain; }
  double ProbLo(int d) const { return problo[d]; }
  double ProbHi(int d) const { return probhi[d]; }
  double CellSize(int d) const { return dx[d]; }
};
struct BCRec {};

template <typename F> void ParallelFor(const Box &b, const F &f) {
  for (int k = b.lo[2]; k <= b.hi[2]; ++k)
    for (int j = b.lo[1]; j <= b.hi[1]; ++j)
      for (int i = b.lo[0]; i <= b.hi[0]; ++i)
        f(i, j, k);
}

class Interpolater {
public:
  virtual ~Interpolater() {}
  virtual Box CoarseBox(const Box &fine, int ratio) = 0;
  virtual Box CoarseBox(const Box &fine, const IntVect &ratio) = 0;
  virtual void interp(const FArrayBox &crse, int crse_comp, FArrayBox &fine,
                      int fine_comp, int ncomp, const Box &fine_region,
                      const IntVect &ratio, const Geometry &crse_geom,
                      const Geometry &fine_geom, Vector<BCRec> const &bcr,
                      int actual_comp, int actual_state, RunOn gpu_or_cpu) = 0;
  virtual void interp_face(const FArrayBox &crse, int crse_comp,
                           FArrayBox &fine, int fine_comp, int ncomp,
                           const Box &fine_region, const IntVect &ratio,
                           const IArrayBox &solve_mask,
                           const Geometry &crse_geom, const Geometry &fine_geom,
                           Vector<BCRec> const &bcr, int bccomp,
                           RunOn gpu_or_cpu) = 0;
};
} // namespace amrex
#endif
