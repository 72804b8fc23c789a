// The (vertex kind, cell kind) pairs of the separable operators in the
// registry, one streaming-kernel instantiation each: interpolate p
// (VC POLY p / CC POLY p), conservative 0 and 1, ddf p (VC POLY p /
// CC CONS p-1), minmod p (VC POLY p / CC MINMOD), hermite and natural p
// (VC POLY p / CC CONS p).  The linear-fallback families are separable only
// where they reduce to one of these pairs.
#pragma once

// X(index, vertex kind type, cell kind type, vertex kind id, cell kind id)
#define CXB_STREAM_PAIRS(X)                                                    \
  X(0, VcPoly<1>, CcPoly<1>, K_VC_POLY1, K_CC_POLY1)                           \
  X(1, VcPoly<3>, CcPoly<3>, K_VC_POLY3, K_CC_POLY3)                           \
  X(2, VcPoly<5>, CcPoly<5>, K_VC_POLY5, K_CC_POLY5)                           \
  X(3, VcPoly<7>, CcPoly<7>, K_VC_POLY7, K_CC_POLY7)                           \
  X(4, VcCons<0>, CcCons<0>, K_VC_CONS0, K_CC_CONS0)                           \
  X(5, VcCons<1>, CcCons<2>, K_VC_CONS1, K_CC_CONS2)                           \
  X(6, VcPoly<1>, CcCons<0>, K_VC_POLY1, K_CC_CONS0)                           \
  X(7, VcPoly<3>, CcCons<2>, K_VC_POLY3, K_CC_CONS2)                           \
  X(8, VcPoly<5>, CcCons<4>, K_VC_POLY5, K_CC_CONS4)                           \
  X(9, VcPoly<7>, CcCons<6>, K_VC_POLY7, K_CC_CONS6)                           \
  X(10, VcPoly<1>, CcMinmod, K_VC_POLY1, K_CC_MINMOD1)                         \
  X(11, VcPoly<3>, CcMinmod, K_VC_POLY3, K_CC_MINMOD1)                         \
  X(12, VcPoly<5>, CcMinmod, K_VC_POLY5, K_CC_MINMOD1)                         \
  X(13, VcPoly<1>, CcCons<1>, K_VC_POLY1, K_CC_CONS1)                          \
  X(14, VcPoly<3>, CcCons<3>, K_VC_POLY3, K_CC_CONS3)                          \
  X(15, VcPoly<5>, CcCons<5>, K_VC_POLY5, K_CC_CONS5)                          \
  X(16, VcPoly<7>, CcCons<7>, K_VC_POLY7, K_CC_CONS7)

namespace cxb {
constexpr int kStreamPairs = 17;
constexpr int kStreamParts = 8; // one file per centring (8 instantiations per pair)
} // namespace cxb
