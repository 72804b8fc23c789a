/* Replaces the bodies of CarpetX/src/driver.hxx and CarpetX/src/timer.hxx for
 * the oracle build.  Their include guards are pre-defined on the command line,
 * so the reference sources compile unmodified against this prelude, which
 * supplies the few names the transfer operators take from those headers. */
#ifndef CX_REF_PRELUDE_HXX
#define CX_REF_PRELUDE_HXX
#include <cctk.h>
#include <AMReX_Interpolater.H>
#include <vect.hxx>
#include <cmath>
#include <mutex>
#include <sstream>
#include <string>
namespace CarpetX {
using namespace Arith;
constexpr int dim = 3;
struct Timer {
  explicit Timer(const std::string &) {}
};
struct Interval {
  explicit Interval(const Timer &) {}
};
} // namespace CarpetX
#endif
