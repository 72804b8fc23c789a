/* Stand-in for the Loop thorn's loop_device.hxx in the oracle build of the
 * reference boundary conditions: only the grid-function view they use.
 * GF3D2layout(imin, imax) addresses the box [imin, imax) Fortran ordered,
 * x fastest, and np is its point count (Loop/src/loop.hxx:926-958);
 * GF3D2 reads and stores one point of such a view. */
#ifndef CX_REF_STUB_LOOP_DEVICE_HXX
#define CX_REF_STUB_LOOP_DEVICE_HXX
#include <vect.hxx>
namespace Loop {
struct GF3D2layout {
  static constexpr int di = 1;
  int dj, dk, np, off;
  GF3D2layout(const Arith::vect<int, 3> &imin, const Arith::vect<int, 3> &imax)
      : dj(imax[0] - imin[0]), dk(dj * (imax[1] - imin[1])), np(dk * (imax[2] - imin[2])),
        off(imin[0] * di + imin[1] * dj + imin[2] * dk) {}
  int linear(const Arith::vect<int, 3> &p) const {
    return p[0] * di + p[1] * dj + p[2] * dk - off;
  }
};
template <typename T> struct GF3D2 {
  GF3D2layout layout;
  T *ptr;
  GF3D2(const GF3D2layout &l, T *p) : layout(l), ptr(p) {}
  T &operator()(const Arith::vect<int, 3> &p) const { return ptr[layout.linear(p)]; }
  void store(const Arith::vect<int, 3> &p, const T &v) const { ptr[layout.linear(p)] = v; }
};
} // namespace Loop
#endif
