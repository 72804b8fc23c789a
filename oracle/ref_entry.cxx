/* C entry points over the reference transfer operators, compiled unmodified
 * from CarpetX/src/prolongate_3d_rf2*.cxx.  Test infrastructure only: this is
 * the oracle the CUDA path is checked against, never part of the product.
 *
 * The type-name -> operator-table mapping restates get_interpolator
 * (CarpetX/src/driver.cxx:593-628); indextype = (ix<<2)|(iy<<1)|iz
 * (driver.cxx:595-596). */
#include "prolongate_3d_rf2.hxx"

#include <cstring>
#include <map>
#include <string>

int cx_ref_prolongate_per_group = 0;

namespace {
const std::map<int, std::array<amrex::Interpolater *, 8> > *
table_for(const char *type) {
  using namespace CarpetX;
  const std::string t(type);
  if (t == "interpolate")
    return &prolongate_poly_3d_rf2;
  if (t == "conservative")
    return &prolongate_cons_3d_rf2;
  if (t == "ddf")
    return &prolongate_ddf_3d_rf2;
  if (t == "eno")
    return &prolongate_eno_3d_rf2;
  if (t == "minmod")
    return &prolongate_minmod_3d_rf2;
  if (t == "hermite")
    return &prolongate_hermite_3d_rf2;
  if (t == "natural")
    return &prolongate_natural_3d_rf2;
  if (t == "poly-cons3lfb")
    return &prolongate_poly_cons3lfb_3d_rf2;
  if (t == "poly-eno3lfb")
    return &prolongate_poly_eno3lfb_3d_rf2;
  return nullptr;
}

amrex::Interpolater *lookup(const char *type, int order, int indextype) {
  const auto *tab = table_for(type);
  if (!tab || indextype < 0 || indextype > 7 || tab->count(order) == 0)
    return nullptr;
  return tab->at(order).at(indextype);
}

amrex::Box mkbox(const int *lo, const int *hi) {
  return amrex::Box(amrex::IntVect(lo[0], lo[1], lo[2]),
                    amrex::IntVect(hi[0], hi[1], hi[2]));
}
} // namespace

extern "C" {

/* 0 if (type, order, indextype) names a reference operator, else -1. */
int ref_prolong_exists(const char *type, int order, int indextype) {
  return lookup(type, order, indextype) ? 0 : -1;
}

/* CoarseBox(fine) of the operator (impl.hxx:1236-1254). */
int ref_coarse_box(const char *type, int order, int indextype,
                   const int fine_lo[3], const int fine_hi[3], int crse_lo[3],
                   int crse_hi[3]) {
  amrex::Interpolater *op = lookup(type, order, indextype);
  if (!op)
    return -1;
  const amrex::Box c = op->CoarseBox(mkbox(fine_lo, fine_hi), 2);
  for (int d = 0; d < 3; ++d) {
    crse_lo[d] = c.lo[d];
    crse_hi[d] = c.hi[d];
  }
  return 0;
}

/* Runs the reference interp() on n boxes, one OpenMP task per box (the
 * reference parallelises over boxes/tiles with OpenMP around interp, as
 * AMReX's MFIter does).  Arrays are indexed per box; boxes are 3 ints each.
 * Used for the CPU-baseline timing. */
int ref_prolong_many(int n, const char *const *types, const int *orders,
                     const int *indextypes, int per_group,
                     const double *const *crse, const int *crse_lo,
                     const int *crse_hi, double *const *fine,
                     const int *fine_lo, const int *fine_hi, const int *reg_lo,
                     const int *reg_hi, const int *ncomp) {
  for (int b = 0; b < n; ++b)
    if (!lookup(types[b], orders[b], indextypes[b]))
      return -1;
  cx_ref_prolongate_per_group = per_group;
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < n; ++b) {
    amrex::Interpolater *op = lookup(types[b], orders[b], indextypes[b]);
    amrex::FArrayBox cfab(mkbox(crse_lo + 3 * b, crse_hi + 3 * b),
                          const_cast<double *>(crse[b]), ncomp[b]);
    amrex::FArrayBox ffab(mkbox(fine_lo + 3 * b, fine_hi + 3 * b), fine[b],
                          ncomp[b]);
    const amrex::Vector<amrex::BCRec> bcr;
    op->interp(cfab, 0, ffab, 0, ncomp[b],
               mkbox(reg_lo + 3 * b, reg_hi + 3 * b), amrex::IntVect(2, 2, 2),
               amrex::Geometry(), amrex::Geometry(), bcr, 0, 0,
               amrex::RunOn::Cpu);
  }
  return 0;
}

/* Runs the reference interp() (impl.hxx:2167-2188) on host FABs.  crse/fine
 * hold ncomp components, each of box.numPts() doubles, x fastest. */
int ref_prolong(const char *type, int order, int indextype, int per_group,
                const double *crse, const int crse_lo[3], const int crse_hi[3],
                double *fine, const int fine_lo[3], const int fine_hi[3],
                const int reg_lo[3], const int reg_hi[3], int ncomp) {
  amrex::Interpolater *op = lookup(type, order, indextype);
  if (!op)
    return -1;
  cx_ref_prolongate_per_group = per_group;
  amrex::FArrayBox cfab(mkbox(crse_lo, crse_hi), const_cast<double *>(crse),
                        ncomp);
  amrex::FArrayBox ffab(mkbox(fine_lo, fine_hi), fine, ncomp);
  const amrex::Vector<amrex::BCRec> bcr;
  op->interp(cfab, 0, ffab, 0, ncomp, mkbox(reg_lo, reg_hi),
             amrex::IntVect(2, 2, 2), amrex::Geometry(), amrex::Geometry(),
             bcr, 0, 0, amrex::RunOn::Cpu);
  return 0;
}
}
