/* Stand-in for <AMReX.H> in the oracle build of the reference boundary
 * conditions (CarpetX/src/boundaries.cxx): the types live in the
 * Interpolater stand-in. */
#ifndef CX_REF_STUB_AMREX_H
#define CX_REF_STUB_AMREX_H
#include <AMReX_Interpolater.H>
#endif
