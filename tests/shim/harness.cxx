// Test harness: drives the amrex::Interpolater shim
// (carpetx_b200/host/prolongate_3d_rf2_b200.cxx) through the registration
// tables and the virtual base-class interface, as CarpetX's fill-patch code
// does, compiled against the oracle's AMReX/Cactus stand-in headers.
#include "prolongate_3d_rf2_b200.hxx"

#include <string>

int cx_ref_prolongate_per_group = 0; // CarpetX parameter prolongate_per_group

namespace {
// type name -> table, as get_interpolator (CarpetX/src/driver.cxx:602-627)
amrex::Interpolater *lookup(const char *type, int order, int indextype) {
  using namespace CarpetX;
  const std::string t(type);
  const std::map<int, std::array<amrex::Interpolater *, 8> > *ops =
      t == "interpolate"     ? &prolongate_poly_3d_rf2
      : t == "conservative"  ? &prolongate_cons_3d_rf2
      : t == "ddf"           ? &prolongate_ddf_3d_rf2
      : t == "eno"           ? &prolongate_eno_3d_rf2
      : t == "minmod"        ? &prolongate_minmod_3d_rf2
      : t == "hermite"       ? &prolongate_hermite_3d_rf2
      : t == "natural"       ? &prolongate_natural_3d_rf2
      : t == "poly-cons3lfb" ? &prolongate_poly_cons3lfb_3d_rf2
      : t == "poly-eno3lfb"  ? &prolongate_poly_eno3lfb_3d_rf2
                             : nullptr;
  if (!ops || !ops->count(order) || indextype < 0 || indextype > 7)
    return nullptr;
  return ops->at(order).at(indextype);
}
amrex::Box mkbox(const int *lo, const int *hi) {
  return amrex::Box(amrex::IntVect(lo[0], lo[1], lo[2]),
                    amrex::IntVect(hi[0], hi[1], hi[2]));
}
} // namespace

extern "C" int shim_coarse_box(const char *type, int order, int indextype,
                               const int flo[3], const int fhi[3], int clo[3],
                               int chi[3]) {
  amrex::Interpolater *op = lookup(type, order, indextype);
  if (!op)
    return -1;
  const amrex::Box c = op->CoarseBox(mkbox(flo, fhi), 2);
  for (int d = 0; d < 3; ++d) {
    clo[d] = c.lo[d];
    chi[d] = c.hi[d];
  }
  return 0;
}

// crse / fine are device pointers (an AMReX GPU build's FAB memory).
extern "C" int shim_interp(const char *type, int order, int indextype,
                           int per_group, double *crse, const int clo[3],
                           const int chi[3], double *fine, const int flo[3],
                           const int fhi[3], const int rlo[3], const int rhi[3],
                           int ncomp, int face) {
  amrex::Interpolater *op = lookup(type, order, indextype);
  if (!op)
    return -1;
  cx_ref_prolongate_per_group = per_group;
  amrex::FArrayBox cfab(mkbox(clo, chi), crse, ncomp);
  amrex::FArrayBox ffab(mkbox(flo, fhi), fine, ncomp);
  const amrex::Vector<amrex::BCRec> bcr;
  if (face)
    op->interp_face(cfab, 0, ffab, 0, ncomp, mkbox(rlo, rhi),
                    amrex::IntVect(2, 2, 2), amrex::IArrayBox(),
                    amrex::Geometry(), amrex::Geometry(), bcr, 0,
                    amrex::RunOn::Gpu);
  else
    op->interp(cfab, 0, ffab, 0, ncomp, mkbox(rlo, rhi),
               amrex::IntVect(2, 2, 2), amrex::Geometry(), amrex::Geometry(),
               bcr, 0, 0, amrex::RunOn::Gpu);
  return 0;
}
