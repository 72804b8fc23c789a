/* Replaces the body of CarpetX/src/driver.hxx for the oracle build of the
 * reference boundary conditions (CarpetX/src/boundaries*.cxx), whose include
 * guard is pre-defined on the command line: the symmetry and boundary enums
 * (driver.hxx:41-57), and the few members of GHExt, PatchData and GroupData
 * that BoundaryCondition reads (driver.hxx:347-351, 397-411, 486). */
#ifndef CX_REF_BC_PRELUDE_HXX
#define CX_REF_BC_PRELUDE_HXX
#include <cctk.h>
#include <AMReX_Interpolater.H>
#include <vect.hxx>
#include <array>
#include <cassert>
#include <cmath>
#include <memory>
#include <vector>
namespace CarpetX {
using namespace Arith;
constexpr int dim = 3;
enum class symmetry_t { none, interpatch, periodic, reflection };
enum class boundary_t { none, symmetry_boundary, dirichlet, linear_extrapolation, neumann, robin };
struct CactusAmrCore {
  amrex::Geometry geom;
  const amrex::Geometry &Geom(int) const { return geom; }
};
struct GHExt {
  struct PatchData {
    std::array<std::array<symmetry_t, dim>, 2> symmetries;
    std::unique_ptr<CactusAmrCore> amrcore;
    struct LevelData {
      struct GroupData {
        int patch, level;
        std::array<int, dim> indextype;
        std::array<std::array<boundary_t, dim>, 2> boundaries;
        std::vector<std::array<int, dim> > parities;
        std::vector<CCTK_REAL> dirichlet_values;
        std::vector<CCTK_REAL> robin_values;
      };
    };
  };
  std::vector<PatchData> patchdata;
};
extern std::unique_ptr<GHExt> ghext;
} // namespace CarpetX
#endif
