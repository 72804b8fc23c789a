// amrex::Interpolater shim over the carpetx_b200 C ABI.
//
// Drop-in replacement for CarpetX's prolongate_3d_rf2<...> operator objects
// (CarpetX/src/prolongate_3d_rf2.hxx:33-120): same base class, same virtual
// interface, same registration tables (prolongate_3d_rf2.hxx:127-177), so
// get_interpolator (CarpetX/src/driver.cxx:593-642) and the fill-patch callers
// (CarpetX/src/fillpatch.cxx:116-119, 179-180, 213-216) work unchanged.  Each
// interp() enqueues one sm_100a kernel on AMReX's current GPU stream and
// returns without synchronising, as the reference's GPU build does
// (impl.hxx:1685-1688).  FAB data must be device memory (an AMReX GPU build).
#ifndef CARPETX_B200_PROLONGATE_3D_RF2_B200_HXX
#define CARPETX_B200_PROLONGATE_3D_RF2_B200_HXX

#include <AMReX_Interpolater.H>

#include <array>
#include <map>

#include "carpetx_b200.h"

namespace CarpetX {

class prolongate_3d_rf2_b200 final : public amrex::Interpolater {
  cx_op_t op_;

public:
  // (prolongation_type, prolongation_order, indextype) as in
  // get_interpolator; an unknown operator is a CCTK_VERROR, as there
  // (driver.cxx:621-625).
  prolongate_3d_rf2_b200(const char *type, int order, int indextype);
  virtual ~prolongate_3d_rf2_b200() override;

  // coarsen(fine, 2) grown by the stencil's required ghosts
  // (impl.hxx:1226-1254); ratio must be 2.
  virtual amrex::Box CoarseBox(const amrex::Box &fine, int ratio) override;
  virtual amrex::Box CoarseBox(const amrex::Box &fine,
                               const amrex::IntVect &ratio) override;

  // impl.hxx:2167-2188: per var or per group by the CarpetX parameter
  // prolongate_per_group; asserts ratio == 2, actual_comp == 0,
  // actual_state == 0 and fine_region inside fine.box(), as the reference.
  virtual void interp(const amrex::FArrayBox &crse, int crse_comp,
                      amrex::FArrayBox &fine, int fine_comp, int ncomp,
                      const amrex::Box &fine_region,
                      const amrex::IntVect &ratio,
                      const amrex::Geometry &crse_geom,
                      const amrex::Geometry &fine_geom,
                      amrex::Vector<amrex::BCRec> const &bcr, int actual_comp,
                      int actual_state, amrex::RunOn gpu_or_cpu) override;

  // impl.hxx:2190-2208: ignores solve_mask, requires bccomp == 0, forwards.
  virtual void interp_face(const amrex::FArrayBox &crse, int crse_comp,
                           amrex::FArrayBox &fine, int fine_comp, int ncomp,
                           const amrex::Box &fine_region,
                           const amrex::IntVect &ratio,
                           const amrex::IArrayBox &solve_mask,
                           const amrex::Geometry &crse_geom,
                           const amrex::Geometry &fine_geom,
                           amrex::Vector<amrex::BCRec> const &bcr,
                           int bccomp, amrex::RunOn gpu_or_cpu) override;

  cx_op_t op() const { return op_; }
};

// The nine registration tables of prolongate_3d_rf2.hxx:127-177, filled with
// shim objects: order -> operator per indextype (cx<<2 | cy<<1 | cz).
extern const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_poly_3d_rf2;
extern const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_cons_3d_rf2;
extern const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_ddf_3d_rf2;
extern const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_natural_3d_rf2;
extern const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_eno_3d_rf2;
extern const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_minmod_3d_rf2;
extern const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_hermite_3d_rf2;
extern const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_poly_cons3lfb_3d_rf2;
extern const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_poly_eno3lfb_3d_rf2;

} // namespace CarpetX

#endif
