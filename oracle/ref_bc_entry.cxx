/* C entry point into the reference boundary conditions, compiled unmodified
 * from CarpetX/src/boundaries*.cxx (see Makefile).  TEST INFRASTRUCTURE ONLY:
 * the tests call it to pin the C restatement (cx_oracle.c, cxo_boundary_box)
 * and, through it, the CUDA kernels.
 *
 * ref_boundary_box sets up the one patch, level and group that
 * BoundaryCondition reads (symmetries, geometry, boundaries, parities,
 * Dirichlet and Robin values), wraps the caller's array as the destination
 * FArrayBox and runs BoundaryCondition(groupdata, dest).apply()
 * (boundaries.cxx:32-118), as GroupData::apply_boundary_conditions
 * (driver.cxx:967-995) does for each FArrayBox of a MultiFab. */
#include "boundaries.hxx"

#include <memory>

namespace CarpetX {
std::unique_ptr<GHExt> ghext;
}

using namespace CarpetX;

extern "C" int ref_boundary_box(const int symmetry[6], const int boundary[6],
                                const int domain_lo[3], const int domain_hi[3],
                                const double prob_lo[3], const double prob_hi[3],
                                const double dx[3], const int indextype[3], int ncomp,
                                const double *dirichlet, const double *robin,
                                const int *parity, double *data, const int lo[3],
                                const int hi[3]) {
  if (ncomp < 1 || ncomp > 16)
    return -1;
  ghext = std::make_unique<GHExt>();
  ghext->patchdata.resize(1);
  GHExt::PatchData &pd = ghext->patchdata[0];
  pd.amrcore = std::make_unique<CactusAmrCore>();
  amrex::Geometry &geom = pd.amrcore->geom;
  geom.domain = amrex::Box(amrex::IntVect(domain_lo[0], domain_lo[1], domain_lo[2]),
                           amrex::IntVect(domain_hi[0], domain_hi[1], domain_hi[2]));
  for (int d = 0; d < 3; ++d) {
    geom.problo[d] = prob_lo[d];
    geom.probhi[d] = prob_hi[d];
    geom.dx[d] = dx[d];
  }
  GHExt::PatchData::LevelData::GroupData gd;
  gd.patch = 0;
  gd.level = 0;
  for (int f = 0; f < 2; ++f)
    for (int d = 0; d < 3; ++d) {
      pd.symmetries[f][d] = symmetry_t(symmetry[3 * f + d]);
      gd.boundaries[f][d] = boundary_t(boundary[3 * f + d]);
    }
  for (int d = 0; d < 3; ++d)
    gd.indextype[d] = indextype[d];
  for (int c = 0; c < ncomp; ++c) {
    gd.dirichlet_values.push_back(dirichlet[c]);
    gd.robin_values.push_back(robin[c]);
    gd.parities.push_back({parity[3 * c], parity[3 * c + 1], parity[3 * c + 2]});
  }
  amrex::Box box(amrex::IntVect(lo[0], lo[1], lo[2]), amrex::IntVect(hi[0], hi[1], hi[2]));
  for (int d = 0; d < 3; ++d)
    box.typ[d] = indextype[d] ? amrex::IndexType::CELL : amrex::IndexType::NODE;
  amrex::FArrayBox dest(box, data, ncomp);
  BoundaryCondition(gd, dest).apply();
  ghext.reset();
  return 0;
}
