// Transpose of the separable linear prolongations, gather form (no atomics).
//
// A fine point f with offset off reads coarse point floor(f/2) + o with 1-D
// weight w(off, o), o in stencil_radius(off).  Hence coarse point c receives
// from the fine points f = 2 (c - o) + off of the region, and
//   crse_bar(c) = sum_z sum_y sum_x wz * wy * wx * fine_bar(fx, fy, fz).
// One thread per coarse point of the coarse box (every coarse point is
// written, zero where no region point reads it).  The sums run in a fixed
// order, so the result is deterministic.
#include "cx_internal.h"
#include "cx_stencils.cuh"

namespace cxb {
namespace {

// 1-D weight of coarse offset o for a fine point with offset off: the
// coefficient multiplying v[o] in the kind's linear form.
template <class K> struct Weight;

template <int P> struct Weight<VcPoly<P>> {
  __device__ static double w(int off, int o) {
    if (off == 0)
      return o == 0 ? 1.0 : 0.0;
    constexpr int i0 = (P + 1) / 2 - 1;
    if (o < -i0 || o > P - i0)
      return 0.0;
    return vc_poly_c<P>(o + i0); // symmetric pairs share c(i) = c(P - i)
  }
};
template <int P> struct Weight<CcPoly<P>> {
  __device__ static double w(int off, int o) {
    constexpr int I0 = (P + 1) / 2;
    if (off == 0) {
      const int i = o + I0;
      return i >= 0 && i <= P ? cc_poly_c<P>(i) : 0.0;
    }
    const int i = o + I0 - P % 2;
    return i >= 0 && i <= P ? cc_poly_c<P>(P - i) : 0.0;
  }
};
template <int P> struct Weight<CcCons<P>> {
  __device__ static double w(int off, int o) {
    constexpr int I0 = (P + 1) / 2;
    if constexpr (P % 2 == 0) {
      if (o == 0)
        return cc_cons_c<P>(P / 2);
      if (o < -P / 2 || o > P / 2)
        return 0.0;
      const double c = o < 0 ? cc_cons_c<P>(o + I0) : cc_cons_c<P>(P - o - I0);
      const double sgn = (o < 0) == (off == 0) ? 1.0 : -1.0;
      return sgn * c;
    } else {
      if (off == 0) {
        const int i = o + I0;
        return i >= 0 && i <= P ? cc_cons_c<P>(i) : 0.0;
      }
      const int i = (P + 1) / 2 - o;
      return i >= 0 && i <= P ? cc_cons_c<P>(i) : 0.0;
    }
  }
};
template <int P> struct Weight<VcCons<P>> {
  __device__ static double w(int off, int o) {
    if (off == 0)
      return o == 0 ? 1.0 : 0.0;
    if (P == 0)
      return 0.0;
    return o == 0 || o == 1 ? 0.5 : 0.0;
  }
};
template <> struct Weight<CcMinmod> {
  __device__ static double w(int, int) { return 0.0; } // nonlinear: not used
};

template <class K> __device__ __forceinline__ void weight_of(int off, int o, double &w) {
  w = Weight<K>::w(off, o);
}

__device__ __forceinline__ double w1d(int kind, int off, int o) {
  double w = 0.0;
  CXB_DISPATCH_SEPARABLE(kind, weight_of, off, o, w);
  return w;
}

__global__ void __launch_bounds__(256) adjoint_direct_kernel(const BoxDesc b, double *crse_bar) {
  const int64_t cnp = b.cnp;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= cnp)
    return;
  const int comp = blockIdx.y;
  const int c[3] = {b.clo[0] + (int)(idx % b.cnx), b.clo[1] + (int)((idx / b.cnx) % b.cny),
                    b.clo[2] + (int)(idx / ((int64_t)b.cnx * b.cny))};
  const double *g = b.fine + comp * b.fnp; // fine_bar
  const int64_t fplane = (int64_t)b.fnx * b.fny;
  double acc = 0.0;
  for (int offz = 0; offz < 2; ++offz) {
    const KindInfo kz = kind_info(b.kind[2]);
    const int zlo = offz ? kz.r1lo : kz.r0lo, zhi = offz ? kz.r1hi : kz.r0hi;
    for (int oz = zlo; oz <= zhi; ++oz) {
      const int fz = 2 * (c[2] - oz) + offz;
      if (fz < b.rlo[2] || fz > b.rhi[2])
        continue;
      const double wz = w1d(b.kind[2], offz, oz);
      for (int offy = 0; offy < 2; ++offy) {
        const KindInfo ky = kind_info(b.kind[1]);
        const int ylo = offy ? ky.r1lo : ky.r0lo, yhi = offy ? ky.r1hi : ky.r0hi;
        for (int oy = ylo; oy <= yhi; ++oy) {
          const int fy = 2 * (c[1] - oy) + offy;
          if (fy < b.rlo[1] || fy > b.rhi[1])
            continue;
          const double wzy = fmul(wz, w1d(b.kind[1], offy, oy));
          const double *grow = g + (fy - b.flo[1]) * (int64_t)b.fnx + fplane * (fz - b.flo[2]) - b.flo[0];
          for (int offx = 0; offx < 2; ++offx) {
            const KindInfo kx = kind_info(b.kind[0]);
            const int xlo = offx ? kx.r1lo : kx.r0lo, xhi = offx ? kx.r1hi : kx.r0hi;
            for (int ox = xlo; ox <= xhi; ++ox) {
              const int fx = 2 * (c[0] - ox) + offx;
              if (fx < b.rlo[0] || fx > b.rhi[0])
                continue;
              acc = fadd(acc, fmul(fmul(wzy, w1d(b.kind[0], offx, ox)), __ldg(grow + fx)));
            }
          }
        }
      }
    }
  }
  crse_bar[comp * cnp + idx] = acc;
}

} // namespace

cudaError_t launch_prolong_adjoint_box(const BoxDesc &b, int per_group, double *crse_bar,
                                       cudaStream_t s) {
  (void)per_group;
  if (b.ncomp <= 0 || b.cnp <= 0)
    return cudaSuccess;
  dim3 grid((unsigned)((b.cnp + 255) / 256), b.ncomp);
  adjoint_direct_kernel<<<grid, 256, 0, s>>>(b, crse_bar);
  return cudaGetLastError();
}

} // namespace cxb
