// Device 1-D stencils, one struct per kind.
//
// Each struct applies the reference's interp1d<...> (CarpetX/src/
// prolongate_3d_rf2_impl.hxx:396-878) with the reference's association order,
// every product and sum rounded separately (__dmul_rn / __dadd_rn: no FMA
// contraction), so that results equal the host build of the reference as FP64
// values.  Two exact simplifications: the reference starts its sums from
// y = 0 and adds the first product (0 + p = p, except that 0 + (-0) = +0), and
// multiplies by the coefficient 1 (exact); both are skipped, so only the sign
// of an exact-zero result can differ.  `v` points at the value of coarse
// offset 0 of the fine point; OFF is the fine point's offset within its
// coarse cell.
//   RLO/RHI: union over OFF of the stencil radius (window the passes stage).
#pragma once
#include "cx_kinds.h"
#include "stencils_gen.h"

namespace cxb {

__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }

template <int P> CXB_HD constexpr double vc_poly_c(int i) {
  return P == 1 ? kVcPoly1(i) : P == 3 ? kVcPoly3(i) : P == 5 ? kVcPoly5(i) : kVcPoly7(i);
}
template <int P> CXB_HD constexpr double cc_poly_c(int i) {
  return P == 1 ? kCcPoly1(i) : P == 3 ? kCcPoly3(i) : P == 5 ? kCcPoly5(i) : kCcPoly7(i);
}
template <int P> CXB_HD constexpr double cc_cons_c(int i) {
  return P == 0   ? kCcCons0(i)
         : P == 1 ? kCcCons1(i)
         : P == 2 ? kCcCons2(i)
         : P == 3 ? kCcCons3(i)
         : P == 4 ? kCcCons4(i)
         : P == 5 ? kCcCons5(i)
         : P == 6 ? kCcCons6(i)
                  : kCcCons7(i);
}
CXB_HD constexpr double cc_eno2_c(int row, int i) {
  return row == 0 ? kCcEno2Row0(i) : row == 1 ? kCcEno2Row1(i) : kCcEno2Row2(i);
}

// VC POLY p and VC HERMITE p: impl.hxx:411-456, 533-578.
// off 0 injects; off 1 sums symmetric pairs cs[i] * (v[i-i0] + v[p-i-i0]).
template <int P> struct VcPoly {
  static constexpr int KIND = P == 1 ? K_VC_POLY1 : P == 3 ? K_VC_POLY3 : P == 5 ? K_VC_POLY5 : K_VC_POLY7;
  static constexpr int RLO = -((P - 1) / 2), RHI = (P + 1) / 2;
  template <int OFF> __device__ __forceinline__ static double ap(const double *v) {
    if constexpr (OFF == 0) {
      return v[0];
    } else {
      constexpr int N = P + 1, i0 = N / 2 - 1;
      double y = fmul(vc_poly_c<P>(0), fadd(v[-i0], v[P - i0]));
#pragma unroll
      for (int i = 1; i < N / 2; ++i)
        y = fadd(y, fmul(vc_poly_c<P>(i), fadd(v[i - i0], v[P - i - i0])));
      return y;
    }
  }
};

// CC POLY p: impl.hxx:478-511.
template <int P> struct CcPoly {
  static constexpr int KIND = P == 1 ? K_CC_POLY1 : P == 3 ? K_CC_POLY3 : P == 5 ? K_CC_POLY5 : K_CC_POLY7;
  static constexpr int N = P + 1, I0 = N / 2;
  static constexpr int RLO = -I0, RHI = N - 1 - I0 + P % 2;
  template <int OFF> __device__ __forceinline__ static double ap(const double *v) {
    double y = OFF == 0 ? fmul(cc_poly_c<P>(0), v[-I0]) : fmul(cc_poly_c<P>(P), v[-I0 + P % 2]);
#pragma unroll
    for (int i = 1; i < N; ++i) {
      if constexpr (OFF == 0)
        y = fadd(y, fmul(cc_poly_c<P>(i), v[i - I0]));
      else
        y = fadd(y, fmul(cc_poly_c<P>(P - i), v[i - I0 + P % 2]));
    }
    return y;
  }
};

// CC CONS p: impl.hxx:651-715.  Even p: centre tap plus antisymmetric pairs
// (conservative for any data); odd p: plain sums, mirrored for off 1.
template <int P> struct CcCons {
  static constexpr int KIND = K_CC_CONS0 + P;
  static constexpr int N = P + 1, I0 = N / 2;
  static constexpr int RLO = -((P + 1) / 2), RHI = (P + 1) / 2;
  template <int OFF> __device__ __forceinline__ static double ap(const double *v) {
    double y;
    if constexpr (P % 2 == 0) {
      static_assert(cc_cons_c<P>(P / 2) == 1.0, "even conservative stencils have centre weight 1");
      y = v[P / 2 - I0];
#pragma unroll
      for (int i = 0; i < P / 2; ++i) {
        if constexpr (OFF == 0)
          y = fadd(y, fmul(cc_cons_c<P>(i), fsub(v[i - I0], v[P - i - I0])));
        else
          y = fadd(y, fmul(cc_cons_c<P>(i), fsub(v[P - i - I0], v[i - I0])));
      }
    } else {
      y = OFF == 0 ? fmul(cc_cons_c<P>(0), v[-I0]) : fmul(cc_cons_c<P>(0), v[(P + 1) / 2]);
#pragma unroll
      for (int i = 1; i < N; ++i) {
        if constexpr (OFF == 0)
          y = fadd(y, fmul(cc_cons_c<P>(i), v[i - I0]));
        else
          y = fadd(y, fmul(cc_cons_c<P>(i), v[(P + 1) / 2 - i]));
      }
    }
    return y;
  }
};

// Deprecated VC CONS p (p = 0, 1): impl.hxx:603-630.  For p = 0 the off-1
// stencil is empty and the result is 0 (used by "conservative" order 0).
template <int P> struct VcCons {
  static constexpr int KIND = P == 0 ? K_VC_CONS0 : K_VC_CONS1;
  static constexpr int RLO = 0, RHI = P == 0 ? 0 : 1;
  template <int OFF> __device__ __forceinline__ static double ap(const double *v) {
    if constexpr (OFF == 0) {
      return v[0];
    } else if constexpr (P == 0) {
      return 0.0;
    } else {
      return fadd(fmul(0.5, v[0]), fmul(0.5, v[1]));
    }
  }
};

// CC MINMOD 1: impl.hxx:859-877.
struct CcMinmod {
  static constexpr int KIND = K_CC_MINMOD1;
  static constexpr int RLO = -1, RHI = 1;
  template <int OFF> __device__ __forceinline__ static double ap(const double *v) {
    const double cval = v[0];
    const double dm = fsub(cval, v[-1]);
    const double dp = fsub(v[1], cval);
    const double delta = fmul(fadd(copysign(0.125, dm), copysign(0.125, dp)), fmin(fabs(dm), fabs(dp)));
    // cval + sign * delta with sign = -1 (off 0) or +1 (off 1); the product
    // by +-1 is exact
    if constexpr (OFF == 0)
      return fsub(cval, delta);
    else
      return fadd(cval, delta);
  }
};

// Runtime kind -> template dispatch for the separable kinds.
#define CXB_DISPATCH_SEPARABLE(kind, F, ...)                                   \
  switch (kind) {                                                              \
  case K_VC_POLY1: F<VcPoly<1>>(__VA_ARGS__); break;                           \
  case K_VC_POLY3: F<VcPoly<3>>(__VA_ARGS__); break;                           \
  case K_VC_POLY5: F<VcPoly<5>>(__VA_ARGS__); break;                           \
  case K_VC_POLY7: F<VcPoly<7>>(__VA_ARGS__); break;                           \
  case K_VC_CONS0: F<VcCons<0>>(__VA_ARGS__); break;                           \
  case K_VC_CONS1: F<VcCons<1>>(__VA_ARGS__); break;                           \
  case K_CC_POLY1: F<CcPoly<1>>(__VA_ARGS__); break;                           \
  case K_CC_POLY3: F<CcPoly<3>>(__VA_ARGS__); break;                           \
  case K_CC_POLY5: F<CcPoly<5>>(__VA_ARGS__); break;                           \
  case K_CC_POLY7: F<CcPoly<7>>(__VA_ARGS__); break;                           \
  case K_CC_CONS0: F<CcCons<0>>(__VA_ARGS__); break;                           \
  case K_CC_CONS1: F<CcCons<1>>(__VA_ARGS__); break;                           \
  case K_CC_CONS2: F<CcCons<2>>(__VA_ARGS__); break;                           \
  case K_CC_CONS3: F<CcCons<3>>(__VA_ARGS__); break;                           \
  case K_CC_CONS4: F<CcCons<4>>(__VA_ARGS__); break;                           \
  case K_CC_CONS5: F<CcCons<5>>(__VA_ARGS__); break;                           \
  case K_CC_CONS6: F<CcCons<6>>(__VA_ARGS__); break;                           \
  case K_CC_CONS7: F<CcCons<7>>(__VA_ARGS__); break;                           \
  case K_CC_MINMOD1: F<CcMinmod>(__VA_ARGS__); break;                          \
  default: break;                                                              \
  }


} // namespace cxb
