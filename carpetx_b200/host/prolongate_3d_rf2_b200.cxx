// amrex::Interpolater shim over the carpetx_b200 C ABI (see the header).
// Replaces CarpetX/src/prolongate_3d_rf2_impl_*.cxx in a CarpetX build.
#include "prolongate_3d_rf2_b200.hxx"

#include <cctk.h>
#include <cctk_Parameters.h>

#include <cassert>
#include <initializer_list>

#ifndef CX_B200_STREAM
#ifdef AMREX_USE_GPU
#include <AMReX_Gpu.H>
#define CX_B200_STREAM() ((cx_stream_t)amrex::Gpu::gpuStream())
#else
#define CX_B200_STREAM() ((cx_stream_t) nullptr)
#endif
#endif

namespace CarpetX {

namespace {
void check(int status, const char *what) {
  if (status != CX_OK)
    CCTK_VERROR("%s: %s (%s)", what, cx_status_string(status), cx_last_error());
}

void box_to(const amrex::Box &b, int lo[3], int hi[3]) {
  for (int d = 0; d < 3; ++d) {
    lo[d] = b.smallEnd()[d];
    hi[d] = b.bigEnd()[d];
  }
}
} // namespace

prolongate_3d_rf2_b200::prolongate_3d_rf2_b200(const char *type, int order,
                                               int indextype) {
  check(cx_prolong_lookup(type, order, indextype, &op_), "prolongation lookup");
}

prolongate_3d_rf2_b200::~prolongate_3d_rf2_b200() {}

amrex::Box prolongate_3d_rf2_b200::CoarseBox(const amrex::Box &fine, int ratio) {
  return CoarseBox(fine, amrex::IntVect(ratio));
}

amrex::Box prolongate_3d_rf2_b200::CoarseBox(const amrex::Box &fine,
                                             const amrex::IntVect &ratio) {
  for (int d = 0; d < 3; ++d)
    assert(ratio[d] == 2);
  int flo[3], fhi[3], clo[3], chi[3];
  box_to(fine, flo, fhi);
  check(cx_prolong_coarse_box(op_, flo, fhi, clo, chi), "CoarseBox");
  return amrex::Box(amrex::IntVect(clo[0], clo[1], clo[2]),
                    amrex::IntVect(chi[0], chi[1], chi[2]));
}

void prolongate_3d_rf2_b200::interp(
    const amrex::FArrayBox &crse, const int crse_comp, amrex::FArrayBox &fine,
    const int fine_comp, const int ncomp, const amrex::Box &fine_region,
    const amrex::IntVect &ratio, const amrex::Geometry &crse_geom,
    const amrex::Geometry &fine_geom, amrex::Vector<amrex::BCRec> const &bcr,
    const int actual_comp, const int actual_state,
    const amrex::RunOn gpu_or_cpu) {
  DECLARE_CCTK_PARAMETERS;
  for (int d = 0; d < 3; ++d)
    assert(ratio[d] == 2);
  assert(actual_comp == 0);
  assert(actual_state == 0);
  int clo[3], chi[3], flo[3], fhi[3], rlo[3], rhi[3];
  box_to(crse.box(), clo, chi);
  box_to(fine.box(), flo, fhi);
  box_to(fine_region, rlo, rhi);
  check(cx_prolong_box(op_, crse.dataPtr(crse_comp), clo, chi,
                       fine.dataPtr(fine_comp), flo, fhi, rlo, rhi, ncomp,
                       prolongate_per_group ? 1 : 0, CX_B200_STREAM()),
        "prolongation");
}

void prolongate_3d_rf2_b200::interp_face(
    const amrex::FArrayBox &crse, const int crse_comp, amrex::FArrayBox &fine,
    const int fine_comp, const int ncomp, const amrex::Box &fine_region,
    const amrex::IntVect &ratio, const amrex::IArrayBox &solve_mask,
    const amrex::Geometry &crse_geom, const amrex::Geometry &fine_geom,
    amrex::Vector<amrex::BCRec> const &bcr, const int bccomp,
    const amrex::RunOn gpu_or_cpu) {
  assert(bccomp == 0);
  interp(crse, crse_comp, fine, fine_comp, ncomp, fine_region, ratio,
         crse_geom, fine_geom, bcr, 0, 0, gpu_or_cpu);
}

namespace {
// One table: for every order, the 8 centrings of (type, order).
std::map<int, std::array<amrex::Interpolater *, 8> >
make_table(const char *type, std::initializer_list<int> orders) {
  std::map<int, std::array<amrex::Interpolater *, 8> > t;
  for (int o : orders) {
    std::array<amrex::Interpolater *, 8> a;
    for (int it = 0; it < 8; ++it)
      a[it] = new prolongate_3d_rf2_b200(type, o, it); // program lifetime
    t.emplace(o, a);
  }
  return t;
}
} // namespace

// Same families and orders as prolongate_3d_rf2_impl_*.cxx
const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_poly_3d_rf2 = make_table("interpolate", {1, 3, 5, 7});
const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_cons_3d_rf2 = make_table("conservative", {0, 1});
const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_ddf_3d_rf2 = make_table("ddf", {1, 3, 5, 7});
const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_natural_3d_rf2 = make_table("natural", {1, 3, 5, 7});
const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_eno_3d_rf2 = make_table("eno", {3, 5});
const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_minmod_3d_rf2 = make_table("minmod", {1, 3, 5});
const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_hermite_3d_rf2 = make_table("hermite", {1, 3, 5});
const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_poly_cons3lfb_3d_rf2 = make_table("poly-cons3lfb", {1, 3, 5});
const std::map<int, std::array<amrex::Interpolater *, 8> >
    prolongate_poly_eno3lfb_3d_rf2 = make_table("poly-eno3lfb", {1, 3, 5});

} // namespace CarpetX
