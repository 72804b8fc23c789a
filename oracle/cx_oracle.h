/* CPU restatement of CarpetX's refinement-factor-2 transfer operators.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; nothing in the product links or calls it.  It follows the
 * reference algorithm point by point (CarpetX/src/prolongate_3d_rf2_impl.hxx)
 * and restates AMReX's average_down family for restriction.
 *
 * Parity status: prolongation is pinned bit-for-bit against the reference
 * operators compiled unmodified (oracle/_ref, see Makefile) and against
 * committed golden fixtures generated from them.  Restriction is
 * "parity unpinned": its arithmetic lives in AMReX (not in the reference
 * tree), so it restates AMReX's published average_down semantics.
 *
 * Layout everywhere: a box is inclusive [lo, hi] per direction; data are
 * Fortran ordered (x fastest) with component stride = number of box points,
 * as in amrex::FArrayBox. */
#ifndef CX_ORACLE_H
#define CX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { CXO_VC = 0, CXO_CC = 1 };
enum { CXO_POLY = 0, CXO_HERMITE = 1, CXO_CONS = 2, CXO_ENO = 3, CXO_MINMOD = 4 };
enum { CXO_FB_NONE = 0, CXO_FB_LINEAR = 1 };

typedef struct {
  int cent[3];  /* CXO_VC / CXO_CC per direction */
  int intp[3];  /* CXO_POLY ... CXO_MINMOD per direction */
  int order[3]; /* per-direction order */
  int fb;       /* CXO_FB_NONE / CXO_FB_LINEAR */
} cxo_op;

/* Operator for (family name, order, indextype) as registered in the nine
 * reference tables (prolongate_3d_rf2_impl_*.cxx) and looked up by
 * get_interpolator (driver.cxx:593-628).  Returns 0, or -1 if unknown. */
int cxo_lookup(const char *type, int order, int indextype, cxo_op *op);

/* interp1d<...>::required_ghosts per direction. */
void cxo_required_ghosts(const cxo_op *op, int ghosts[3]);

/* CoarseBox (impl.hxx:1236-1254): coarsen by 2 (floor), grow by ghosts. */
void cxo_coarse_box(const cxo_op *op, const int fine_lo[3],
                    const int fine_hi[3], int crse_lo[3], int crse_hi[3]);

/* interp() (impl.hxx:2167-2188): per_group selects interp_per_group.
 * shifts (optional, may be NULL) receives the chosen ENO shift per fine point
 * of the region as 3 signed bytes (x,y,z), region points x fastest; in
 * per-var mode one block per component, in per-group mode one block.
 * fallback (optional) receives 1 where FB_LINEAR chose the linear value, same
 * indexing without the factor 3.  Returns 0 or -1 on bad arguments. */
int cxo_prolong(const cxo_op *op, int per_group, const double *crse,
                const int crse_lo[3], const int crse_hi[3], double *fine,
                const int fine_lo[3], const int fine_hi[3],
                const int reg_lo[3], const int reg_hi[3], int ncomp,
                signed char *shifts, unsigned char *fallback);

/* Restriction for a group of the given indextype (bit 2-d set = cell centred
 * in direction d), restating AMReX average_down / _faces / _edges / _nodal as
 * called from Restrict (schedule.cxx:2793-2815): for every coarse point of
 * the coarse region [reg_lo, reg_hi], vertex-centred directions inject the
 * fine point 2c, cell-centred directions average the two children 2c, 2c+1;
 * the children are summed z-outer, x-inner starting from 0 and the sum is
 * scaled by 1/(number of children).  Fully vertex-centred data is a plain
 * copy. */
int cxo_restrict(int indextype, const double *fine, const int fine_lo[3],
                 const int fine_hi[3], double *crse, const int crse_lo[3],
                 const int crse_hi[3], const int reg_lo[3],
                 const int reg_hi[3], int ncomp);

/* Transpose of the prolongation linearised at `crse` (ENO shift, minmod
 * branch and linear-fallback choice taken from the forward input):
 * crse_bar[c] = sum over region fine points f of dP(f)/dc * fine_bar[f].
 * crse_bar is overwritten over its whole box.  Scatter form, plain sums. */
int cxo_prolong_adjoint(const cxo_op *op, int per_group, const double *crse,
                        const int crse_lo[3], const int crse_hi[3],
                        const double *fine_bar, const int fine_lo[3],
                        const int fine_hi[3], const int reg_lo[3],
                        const int reg_hi[3], int ncomp, double *crse_bar);

/* Transpose of cxo_restrict: fine_bar is overwritten over its whole box. */
int cxo_restrict_adjoint(int indextype, const double *crse_bar,
                         const int crse_lo[3], const int crse_hi[3],
                         double *fine_bar, const int fine_lo[3],
                         const int fine_hi[3], const int reg_lo[3],
                         const int reg_hi[3], int ncomp);

/* Outer boundary conditions of one FArrayBox [lo, hi] (ncomp components,
 * at most 16), restating BoundaryCondition(groupdata, dest).apply()
 * (CarpetX/src/boundaries.cxx, boundaries_impl.hxx).  symmetry[3f+d] and
 * boundary[3f+d] are CarpetX's symmetry_t / boundary_t values (driver.hxx:
 * 41-57) of face f (0 lower, 1 upper) in direction d; domain_lo/hi is the
 * level's cell-centred domain box; indextype[d] = 1 for cell centred;
 * parity[3c+d] the reflection parity of component c.  Writes the points
 * outside the domain interior; returns -1 (nothing written) for an invalid
 * condition or a source point outside the box or the interior. */
int cxo_boundary_box(const int symmetry[6], const int boundary[6],
                     const int domain_lo[3], const int domain_hi[3],
                     const double prob_lo[3], const double prob_hi[3],
                     const double dx[3], const int indextype[3], int ncomp,
                     const double *dirichlet, const double *robin,
                     const int *parity, double *data, const int lo[3],
                     const int hi[3]);

/* The 1-D coefficient row used by the oracle for (cent, intp, order), row
 * `row` for ENO (0..order), exact dyadic values; returns the number of
 * coefficients written (0 if the stencil is not defined). */
int cxo_coeffs(int cent, int intp, int order, int row, double *out);

#ifdef __cplusplus
}
#endif
#endif
