// 1-D stencil kinds and the operator encoding shared by host and device code.
//
// An operator of the reference (prolongate_3d_rf2<CENT, INTP, ORDER, FB> per
// direction, CarpetX/src/prolongate_3d_rf2.hxx:33-120) is a triple of 1-D
// stencil kinds plus the fallback flag.  VC HERMITE p uses exactly the VC POLY
// p arithmetic (interp1d<VC,HERMITE,p> reads coeffs1d<VC,POLY,p>,
// impl.hxx:543), so it shares the VC POLY kind.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define CXB_HD __host__ __device__
#else
#define CXB_HD
#endif

namespace cxb {

enum Kind : int {
  K_VC_POLY1 = 0,
  K_VC_POLY3,
  K_VC_POLY5,
  K_VC_POLY7,
  K_VC_CONS0, // deprecated VC CONS (impl.hxx:584-631)
  K_VC_CONS1,
  K_CC_POLY1,
  K_CC_POLY3,
  K_CC_POLY5,
  K_CC_POLY7,
  K_CC_CONS0,
  K_CC_CONS1,
  K_CC_CONS2,
  K_CC_CONS3,
  K_CC_CONS4,
  K_CC_CONS5,
  K_CC_CONS6,
  K_CC_CONS7,
  K_CC_ENO2,
  K_CC_MINMOD1,
  K_COUNT
};

enum Cent : int { VC = 0, CC = 1 };
enum Intp : int { POLY = 0, CONS = 2, ENO = 3, MINMOD = 4 };

struct KindInfo {
  int cent, intp, order;
  // stencil_radius(shift = 0, off) for off = 0, 1 (lo > hi: empty stencil)
  int r0lo, r0hi, r1lo, r1hi;
  int ghosts; // interp1d::required_ghosts
};

CXB_HD constexpr KindInfo kind_info(int k) {
  switch (k) {
  case K_VC_POLY1: return {VC, POLY, 1, 0, 0, 0, 1, 1};
  case K_VC_POLY3: return {VC, POLY, 3, 0, 0, -1, 2, 2};
  case K_VC_POLY5: return {VC, POLY, 5, 0, 0, -2, 3, 3};
  case K_VC_POLY7: return {VC, POLY, 7, 0, 0, -3, 4, 4};
  case K_VC_CONS0: return {VC, CONS, 0, 0, 0, 1, 0, 0};
  case K_VC_CONS1: return {VC, CONS, 1, 0, 0, 0, 1, 1};
  case K_CC_POLY1: return {CC, POLY, 1, -1, 0, 0, 1, 1};
  case K_CC_POLY3: return {CC, POLY, 3, -2, 1, -1, 2, 2};
  case K_CC_POLY5: return {CC, POLY, 5, -3, 2, -2, 3, 3};
  case K_CC_POLY7: return {CC, POLY, 7, -4, 3, -3, 4, 4};
  case K_CC_CONS0: return {CC, CONS, 0, 0, 0, 0, 0, 0};
  case K_CC_CONS1: return {CC, CONS, 1, -1, 0, 0, 1, 1};
  case K_CC_CONS2: return {CC, CONS, 2, -1, 1, -1, 1, 1};
  case K_CC_CONS3: return {CC, CONS, 3, -2, 1, -1, 2, 2};
  case K_CC_CONS4: return {CC, CONS, 4, -2, 2, -2, 2, 2};
  case K_CC_CONS5: return {CC, CONS, 5, -3, 2, -2, 3, 3};
  case K_CC_CONS6: return {CC, CONS, 6, -3, 3, -3, 3, 3};
  case K_CC_CONS7: return {CC, CONS, 7, -4, 3, -3, 4, 4};
  // ENO: radius at shift 0; the shift search reads +-2 (required_ghosts = 2)
  case K_CC_ENO2: return {CC, ENO, 2, -1, 1, -1, 1, 2};
  case K_CC_MINMOD1: return {CC, MINMOD, 1, -1, 1, -1, 1, 1};
  default: return {-1, -1, -1, 0, 0, 0, 0, 0};
  }
}

// Coarse offsets (relative to the coarse cell of a fine point with offset
// `off`) that any part of the operator may read: the stencil radius, the ENO
// search window (+-2) and, for fallback directions, offsets 0 and 1 of the
// slope test (impl.hxx:1613-1615).
CXB_HD inline void read_range(int k, int off, int *lo, int *hi) {
  const KindInfo ki = kind_info(k);
  if (ki.intp == ENO) {
    *lo = -2;
    *hi = 2;
    return;
  }
  int a = off ? ki.r1lo : ki.r0lo, b = off ? ki.r1hi : ki.r0hi;
  if (a > b) { // empty stencil (VC CONS 0, off 1)
    a = 0;
    b = 0;
  }
  *lo = a;
  *hi = b;
}

// Union radius of a separable kind over both fine offsets (host and device):
// the coarse window a pass stages per fine tile.
CXB_HD constexpr int sep_rlo(int k) {
  return k == K_VC_CONS0 ? 0
                         : (kind_info(k).r0lo < kind_info(k).r1lo ? kind_info(k).r0lo
                                                                  : kind_info(k).r1lo);
}
CXB_HD constexpr int sep_rhi(int k) {
  return k == K_VC_CONS0 ? 0
                         : (kind_info(k).r0hi > kind_info(k).r1hi ? kind_info(k).r0hi
                                                                  : kind_info(k).r1hi);
}

// Operator handle: kinds in bits 0-4, 5-9, 10-14, FB_LINEAR in bit 15.
CXB_HD inline int32_t op_encode(int kx, int ky, int kz, int fb) {
  return (int32_t)(kx | (ky << 5) | (kz << 10) | (fb << 15));
}
CXB_HD inline int op_kind(int32_t op, int d) { return (op >> (5 * d)) & 31; }
CXB_HD inline int op_fb(int32_t op) { return (op >> 15) & 1; }

CXB_HD inline bool op_has_eno(int32_t op) {
  return op_kind(op, 0) == K_CC_ENO2 || op_kind(op, 1) == K_CC_ENO2 ||
         op_kind(op, 2) == K_CC_ENO2;
}

// Whether FB_LINEAR can change a value: the reference compiles the fallback
// out unless a conservative direction (CONS or ENO per var, impl.hxx:
// 1535-1538; CONS only per group, impl.hxx:1990-1992) has order > 1.
CXB_HD inline bool op_fb_active(int32_t op, int per_group) {
  if (!op_fb(op))
    return false;
  for (int d = 0; d < 3; ++d) {
    const KindInfo ki = kind_info(op_kind(op, d));
    const bool cons_like =
        per_group ? ki.intp == CONS : (ki.intp == CONS || ki.intp == ENO);
    if (cons_like && ki.order > 1)
      return true;
  }
  return false;
}

// Separable operators are evaluated pass by pass (x, then y, then z), which
// reproduces call_stencil_3d (impl.hxx:1206-1216) exactly: every fine point
// sharing an x (or x and y) position reuses the same 1-D results.
CXB_HD inline bool op_separable(int32_t op, int per_group) {
  return !op_has_eno(op) && !op_fb_active(op, per_group);
}

} // namespace cxb
